// Binned-SAH BVH builder (object splits, and optionally spatial splits) that writes the
// reference GPU two-wide layout.
//
// This is the builder side of the boundary: the reference writes the same layout from its
// SBVH / binned builders through GpuMeshAdapter / GpuTopLevelAdapter
// (src/imbatracer/core/gpu_adapter.cpp:62-143 and 164-276); this file produces that layout from
// our own binned-SAH build (the binning follows Wald 2007, 32 bins, as the reference's
// FastBvhBuilder does, src/imbatracer/core/fast_bvh_builder.h:172), so scenes built here and scenes
// built by the reference go through the same conversion to the 8-wide layout.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "imbart_internal.h"

namespace imbart {
namespace {

constexpr int kBins = 32;
constexpr int kMaxDepth = 96;          // deeper subtrees fall back to median splits
constexpr int kDummyRight = 0x76543210;  // right child of the single-leaf root wrapper

struct Box {
    float lo[3], hi[3];
    void reset() { for (int a = 0; a < 3; ++a) { lo[a] = FLT_MAX; hi[a] = -FLT_MAX; } }
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], b.lo[a]); hi[a] = std::max(hi[a], b.hi[a]); }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
    }
    float half_area() const {
        float d[3];
        for (int a = 0; a < 3; ++a) d[a] = std::max(hi[a] - lo[a], 0.0f);
        return d[0] * (d[1] + d[2]) + d[1] * d[2];
    }
};

struct Prim {
    Box box;
    float c[3];
};

struct Task {
    int begin, end, depth;
    int parent, child;  // link slot in the parent node (-1 for the root)
};

void write_bb(imbart_bbox& bb, const Box& b) {
    bb.lo_x = b.lo[0]; bb.hi_x = b.hi[0];
    bb.lo_y = b.lo[1]; bb.hi_y = b.hi[1];
    bb.lo_z = b.lo[2]; bb.hi_z = b.hi[2];
}

// Finds the best binned-SAH split of refs[begin, end). Returns false to make a leaf.
// On success refs are partitioned and *mid is the first ref of the right side.
bool split(std::vector<int>& refs, const std::vector<Prim>& prims, int begin, int end,
           int leaf_size, int max_sah_leaf, int depth, float traversal_cost, int* mid, Box* lbox,
           Box* rbox) {
    const int count = end - begin;
    if (count <= leaf_size) return false;
    Box cb; cb.reset();
    Box nb; nb.reset();
    for (int i = begin; i < end; ++i) { cb.grow(prims[refs[i]].c); nb.grow(prims[refs[i]].box); }

    int best_axis = -1, best_bin = -1;
    float best_cost = FLT_MAX;
    if (depth < kMaxDepth) {
        for (int axis = 0; axis < 3; ++axis) {
            const float ext = cb.hi[axis] - cb.lo[axis];
            if (!(ext > 0.0f)) continue;
            const float scale = kBins / ext;
            Box bins[kBins]; int counts[kBins];
            for (int b = 0; b < kBins; ++b) { bins[b].reset(); counts[b] = 0; }
            for (int i = begin; i < end; ++i) {
                const Prim& p = prims[refs[i]];
                int b = (int)((p.c[axis] - cb.lo[axis]) * scale);
                b = std::min(std::max(b, 0), kBins - 1);
                bins[b].grow(p.box); counts[b]++;
            }
            float right_area[kBins]; int right_count[kBins];
            Box acc; acc.reset(); int n = 0;
            for (int b = kBins - 1; b > 0; --b) {
                acc.grow(bins[b]); n += counts[b];
                right_area[b] = acc.half_area(); right_count[b] = n;
            }
            acc.reset(); n = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                acc.grow(bins[b]); n += counts[b];
                if (n == 0 || right_count[b + 1] == 0) continue;
                const float cost = n * acc.half_area() + right_count[b + 1] * right_area[b + 1];
                if (cost < best_cost) { best_cost = cost; best_axis = axis; best_bin = b; }
            }
        }
    }

    const float leaf_cost = count * nb.half_area();
    const float split_cost = traversal_cost * nb.half_area() + best_cost;
    if (best_axis >= 0 && !(split_cost < leaf_cost) && count <= max_sah_leaf) return false;

    int m;
    if (best_axis >= 0) {
        const float scale = kBins / (cb.hi[best_axis] - cb.lo[best_axis]);
        auto it = std::partition(refs.begin() + begin, refs.begin() + end, [&](int r) {
            int b = (int)((prims[r].c[best_axis] - cb.lo[best_axis]) * scale);
            b = std::min(std::max(b, 0), kBins - 1);
            return b <= best_bin;
        });
        m = (int)(it - refs.begin());
    } else {
        // All centroids coincide (or the depth limit was hit): split by the median
        // along the widest centroid axis, falling back to index order.
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (cb.hi[a] - cb.lo[a] > cb.hi[axis] - cb.lo[axis]) axis = a;
        m = begin + count / 2;
        std::nth_element(refs.begin() + begin, refs.begin() + m, refs.begin() + end,
                         [&](int a, int b) { return prims[a].c[axis] < prims[b].c[axis]; });
    }
    if (m <= begin || m >= end) m = begin + count / 2;

    lbox->reset(); rbox->reset();
    for (int i = begin; i < m; ++i) lbox->grow(prims[refs[i]].box);
    for (int i = m; i < end; ++i) rbox->grow(prims[refs[i]].box);
    *mid = m;
    return true;
}

// Generic preorder build. `emit_leaf(begin, end)` writes the leaf payload and returns the
// negative child code (~index). Nodes are appended to nodes_out from *n_nodes on.
template <typename EmitLeaf>
int build_generic(std::vector<Prim>& prims, int leaf_size, int max_sah_leaf, float traversal_cost,
                  imbart_node2* nodes_out, int nodes_cap, int* n_nodes, EmitLeaf emit_leaf) {
    const int n = (int)prims.size();
    std::vector<int> refs(n);
    for (int i = 0; i < n; ++i) refs[i] = i;

    Box root_box; root_box.reset();
    for (const Prim& p : prims) root_box.grow(p.box);

    std::vector<Task> stack;
    stack.push_back({0, n, 0, -1, 0});
    std::vector<int> leaf_refs;
    while (!stack.empty()) {
        Task t = stack.back(); stack.pop_back();
        int mid; Box lb, rb;
        const bool inner = split(refs, prims, t.begin, t.end, leaf_size, max_sah_leaf, t.depth, traversal_cost, &mid,
                                 &lb, &rb);
        if (!inner) {
            leaf_refs.assign(refs.begin() + t.begin, refs.begin() + t.end);
            int code;
            const int err = emit_leaf(leaf_refs, &code);
            if (err) return err;
            if (t.parent < 0) {
                // Single-leaf root: wrap it like the reference does (gpu_adapter.cpp:14-31).
                if (*n_nodes >= nodes_cap) return IMBART_ERR_LIMIT;
                imbart_node2& nd = nodes_out[(*n_nodes)++];
                std::memset(&nd, 0, sizeof(nd));
                write_bb(nd.left_bb, root_box);
                nd.right_bb.lo_x = nd.right_bb.lo_y = nd.right_bb.lo_z = 0.0f;
                nd.right_bb.hi_x = nd.right_bb.hi_y = nd.right_bb.hi_z = -0.0f;
                nd.left = code; nd.right = kDummyRight;
            } else {
                (&nodes_out[t.parent].left)[t.child] = code;
            }
            continue;
        }
        if (*n_nodes >= nodes_cap) return IMBART_ERR_LIMIT;
        const int idx = (*n_nodes)++;
        imbart_node2& nd = nodes_out[idx];
        std::memset(&nd, 0, sizeof(nd));
        write_bb(nd.left_bb, lb);
        write_bb(nd.right_bb, rb);
        if (t.parent >= 0) (&nodes_out[t.parent].left)[t.child] = idx;
        // Left first in preorder, as the reference writer does.
        stack.push_back({mid, t.end, t.depth + 1, idx, 1});
        stack.push_back({t.begin, mid, t.depth + 1, idx, 0});
    }
    return 0;
}

// ---------------------------------------------------------------------------------------
// Spatial splits (SBVH, Stich, Friedrich and Dietrich, HPG 2009). A node's references may
// be split at a plane: a triangle straddling the plane goes to both children, each with the
// box of the triangle clipped to its side. Spatial splits are binned over the node's box
// (kSpatialBins per axis, each triangle clipped to every bin it overlaps) and only tried where
// the children of the best object split overlap by more than alpha of the root's area, so
// that trees of well-separated geometry stay object-split (alpha 1e-5 of the mesh box's
// area, the default of the reference's SplitBvhBuilder, src/imbatracer/core/sbvh_builder.h:29-49,
// which the reference's GPU mesh adapter uses, gpu_adapter.cpp:60). The number of references
// is bounded by the caller's budget and output capacity.
// ---------------------------------------------------------------------------------------
constexpr int kSpatialBins = 32;
constexpr float kSpatialAlpha = 1e-5f;

struct Ref {
    int prim;
    Box box;
};

struct Tri3 {
    float v[3][3];
};

// Box of the part of triangle t inside the slab lo <= x[axis] <= hi, intersected with `clip`.
// Intersection points are computed in double and the result is widened by a few ulps, so the
// box never misses a point of the triangle part.
Box clip_triangle(const Tri3& t, int axis, float lo, float hi, const Box& clip) {
    Box b; b.reset();
    for (int i = 0; i < 3; ++i) {
        const float* a = t.v[i];
        const float* c = t.v[(i + 1) % 3];
        if (a[axis] >= lo && a[axis] <= hi) b.grow(a);
        const float planes[2] = {lo, hi};
        for (float pl : planes) {
            if ((a[axis] < pl && c[axis] > pl) || (a[axis] > pl && c[axis] < pl)) {
                const double s = ((double)pl - a[axis]) / ((double)c[axis] - a[axis]);
                float p[3];
                for (int k = 0; k < 3; ++k) p[k] = (float)(a[k] + s * ((double)c[k] - a[k]));
                p[axis] = pl;
                b.grow(p);
            }
        }
    }
    for (int k = 0; k < 3; ++k) {
        if (b.lo[k] > b.hi[k]) continue;   // empty
        if (k != axis) {
            b.lo[k] = std::nextafter(std::nextafter(b.lo[k], -FLT_MAX), -FLT_MAX);
            b.hi[k] = std::nextafter(std::nextafter(b.hi[k], FLT_MAX), FLT_MAX);
        }
        b.lo[k] = std::max(b.lo[k], clip.lo[k]);
        b.hi[k] = std::min(b.hi[k], clip.hi[k]);
    }
    return b;
}

bool box_empty(const Box& b) { return b.lo[0] > b.hi[0] || b.lo[1] > b.hi[1] || b.lo[2] > b.hi[2]; }

struct SbvhBuilder {
    const std::vector<Tri3>& tris;
    int leaf_size, max_sah_leaf;
    float traversal_cost;
    long long max_refs;     // bound on the references in all leaves
    long long refs_used;    // references currently in the build (leaves and pending tasks)
    float root_area;

    // Best object split (binned over reference-box centres). Returns the cost or FLT_MAX.
    float object_split(const std::vector<Ref>& refs, int* axis_out, float* plane_out, Box* l, Box* r) const {
        Box cb; cb.reset();
        for (const Ref& rf : refs) {
            float c[3];
            for (int a = 0; a < 3; ++a) c[a] = 0.5f * (rf.box.lo[a] + rf.box.hi[a]);
            cb.grow(c);
        }
        float best = FLT_MAX;
        for (int axis = 0; axis < 3; ++axis) {
            const float ext = cb.hi[axis] - cb.lo[axis];
            if (!(ext > 0.0f)) continue;
            const float scale = kBins / ext;
            Box bins[kBins]; int counts[kBins];
            for (int b = 0; b < kBins; ++b) { bins[b].reset(); counts[b] = 0; }
            for (const Ref& rf : refs) {
                const float c = 0.5f * (rf.box.lo[axis] + rf.box.hi[axis]);
                int b = std::min(std::max((int)((c - cb.lo[axis]) * scale), 0), kBins - 1);
                bins[b].grow(rf.box); counts[b]++;
            }
            Box racc[kBins]; int rcnt[kBins];
            Box acc; acc.reset(); int n = 0;
            for (int b = kBins - 1; b > 0; --b) { acc.grow(bins[b]); n += counts[b]; racc[b] = acc; rcnt[b] = n; }
            acc.reset(); n = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                acc.grow(bins[b]); n += counts[b];
                if (n == 0 || rcnt[b + 1] == 0) continue;
                const float cost = n * acc.half_area() + rcnt[b + 1] * racc[b + 1].half_area();
                if (cost < best) {
                    best = cost; *axis_out = axis; *l = acc; *r = racc[b + 1];
                    *plane_out = cb.lo[axis] + (b + 1) / scale;   // centres below go left
                }
            }
        }
        return best;
    }

    // Best spatial split (binned over the node box). Returns the cost or FLT_MAX.
    float spatial_split(const std::vector<Ref>& refs, const Box& nb, int* axis_out, float* plane_out) const {
        float best = FLT_MAX;
        for (int axis = 0; axis < 3; ++axis) {
            const float lo = nb.lo[axis], ext = nb.hi[axis] - lo;
            if (!(ext > 0.0f)) continue;
            const float w = ext / kSpatialBins;
            Box bins[kSpatialBins]; int enter[kSpatialBins], leave[kSpatialBins];
            for (int b = 0; b < kSpatialBins; ++b) { bins[b].reset(); enter[b] = 0; leave[b] = 0; }
            for (const Ref& rf : refs) {
                int b0 = std::min(std::max((int)((rf.box.lo[axis] - lo) / w), 0), kSpatialBins - 1);
                int b1 = std::min(std::max((int)((rf.box.hi[axis] - lo) / w), 0), kSpatialBins - 1);
                if (b1 < b0) b1 = b0;
                for (int b = b0; b <= b1; ++b) {
                    const float slo = b == 0 ? -FLT_MAX : lo + b * w;
                    const float shi = b == kSpatialBins - 1 ? FLT_MAX : lo + (b + 1) * w;
                    const Box cl = b0 == b1 ? rf.box : clip_triangle(tris[rf.prim], axis, slo, shi, rf.box);
                    if (!box_empty(cl)) bins[b].grow(cl);
                }
                enter[b0]++; leave[b1]++;
            }
            Box racc[kSpatialBins]; int rcnt[kSpatialBins];
            Box acc; acc.reset(); int n = 0;
            for (int b = kSpatialBins - 1; b > 0; --b) { acc.grow(bins[b]); n += leave[b]; racc[b] = acc; rcnt[b] = n; }
            acc.reset(); n = 0;
            for (int b = 0; b < kSpatialBins - 1; ++b) {
                acc.grow(bins[b]); n += enter[b];
                if (n == 0 || rcnt[b + 1] == 0) continue;
                const float cost = n * acc.half_area() + rcnt[b + 1] * racc[b + 1].half_area();
                if (cost < best) { best = cost; *axis_out = axis; *plane_out = lo + (b + 1) * w; }
            }
        }
        return best;
    }

    // Splits `refs` into l / r; returns false for a leaf.
    bool split(std::vector<Ref>& refs, int depth, std::vector<Ref>& l, std::vector<Ref>& r) {
        const int count = (int)refs.size();
        if (count <= leaf_size) return false;
        Box nb; nb.reset();
        for (const Ref& rf : refs) nb.grow(rf.box);
        int oaxis = -1; float oplane = 0.0f; Box ol, orr;
        float best = depth < kMaxDepth ? object_split(refs, &oaxis, &oplane, &ol, &orr) : FLT_MAX;
        bool spatial = false;
        int saxis = -1; float splane = 0.0f;
        if (oaxis >= 0 && refs_used < max_refs) {
            Box ov;
            for (int a = 0; a < 3; ++a) { ov.lo[a] = std::max(ol.lo[a], orr.lo[a]); ov.hi[a] = std::min(ol.hi[a], orr.hi[a]); }
            if (!box_empty(ov) && ov.half_area() > kSpatialAlpha * root_area) {
                const float sc = spatial_split(refs, nb, &saxis, &splane);
                if (sc < best) { best = sc; spatial = true; }
            }
        }
        const float leaf_cost = count * nb.half_area();
        const float split_cost = traversal_cost * nb.half_area() + best;
        if (oaxis >= 0 && !(split_cost < leaf_cost) && count <= max_sah_leaf) return false;
        l.clear(); r.clear();
        if (spatial) {
            for (const Ref& rf : refs) {
                if (rf.box.hi[saxis] <= splane) { l.push_back(rf); continue; }
                if (rf.box.lo[saxis] >= splane) { r.push_back(rf); continue; }
                const Box lb = clip_triangle(tris[rf.prim], saxis, -FLT_MAX, splane, rf.box);
                const Box rb = clip_triangle(tris[rf.prim], saxis, splane, FLT_MAX, rf.box);
                const bool le = box_empty(lb), re = box_empty(rb);
                if (!le && !re && refs_used < max_refs) {
                    l.push_back({rf.prim, lb});
                    r.push_back({rf.prim, rb});
                    ++refs_used;
                } else if (!le && (re || 0.5f * (rf.box.lo[saxis] + rf.box.hi[saxis]) < splane)) {
                    l.push_back(rf);
                } else {
                    r.push_back(rf);
                }
            }
            if (!l.empty() && !r.empty()) return true;
            l.clear(); r.clear();
        }
        if (oaxis >= 0) {
            for (const Ref& rf : refs)
                (0.5f * (rf.box.lo[oaxis] + rf.box.hi[oaxis]) < oplane ? l : r).push_back(rf);
            if (!l.empty() && !r.empty()) return true;
            l.clear(); r.clear();
        }
        // Coincident centres or the depth limit: median split along the widest axis.
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (nb.hi[a] - nb.lo[a] > nb.hi[axis] - nb.lo[axis]) axis = a;
        std::vector<Ref> s = refs;
        const int m = count / 2;
        std::nth_element(s.begin(), s.begin() + m, s.end(), [&](const Ref& a, const Ref& b) {
            return a.box.lo[axis] + a.box.hi[axis] < b.box.lo[axis] + b.box.hi[axis];
        });
        l.assign(s.begin(), s.begin() + m);
        r.assign(s.begin() + m, s.end());
        return true;
    }
};

struct SbvhTask {
    std::vector<Ref> refs;
    int depth, parent, child;
};

template <typename EmitLeaf>
int build_sbvh(const std::vector<Tri3>& tris, int leaf_size, int max_sah_leaf, float traversal_cost,
               long long max_refs, imbart_node2* nodes_out, int nodes_cap, int* n_nodes, EmitLeaf emit_leaf) {
    const int n = (int)tris.size();
    SbvhBuilder b{tris, leaf_size, max_sah_leaf, traversal_cost, std::max<long long>(max_refs, n), n, 0.0f};
    std::vector<SbvhTask> stack(1);
    stack[0].refs.resize(n);
    Box root_box; root_box.reset();
    for (int i = 0; i < n; ++i) {
        Box bx; bx.reset();
        for (int k = 0; k < 3; ++k) bx.grow(tris[i].v[k]);
        stack[0].refs[i] = {i, bx};
        root_box.grow(bx);
    }
    b.root_area = root_box.half_area();
    stack[0].depth = 0; stack[0].parent = -1; stack[0].child = 0;
    std::vector<int> leaf_prims;
    std::vector<Ref> l, r;
    while (!stack.empty()) {
        SbvhTask t = std::move(stack.back());
        stack.pop_back();
        if (!b.split(t.refs, t.depth, l, r)) {
            leaf_prims.clear();
            for (const Ref& rf : t.refs) leaf_prims.push_back(rf.prim);
            int code;
            const int err = emit_leaf(leaf_prims, &code);
            if (err) return err;
            if (t.parent < 0) {
                if (*n_nodes >= nodes_cap) return IMBART_ERR_LIMIT;
                imbart_node2& nd = nodes_out[(*n_nodes)++];
                std::memset(&nd, 0, sizeof(nd));
                write_bb(nd.left_bb, root_box);
                nd.right_bb.lo_x = nd.right_bb.lo_y = nd.right_bb.lo_z = 0.0f;
                nd.right_bb.hi_x = nd.right_bb.hi_y = nd.right_bb.hi_z = -0.0f;
                nd.left = code; nd.right = kDummyRight;
            } else {
                (&nodes_out[t.parent].left)[t.child] = code;
            }
            continue;
        }
        if (*n_nodes >= nodes_cap) return IMBART_ERR_LIMIT;
        const int idx = (*n_nodes)++;
        imbart_node2& nd = nodes_out[idx];
        std::memset(&nd, 0, sizeof(nd));
        Box lb, rb; lb.reset(); rb.reset();
        for (const Ref& rf : l) lb.grow(rf.box);
        for (const Ref& rf : r) rb.grow(rf.box);
        write_bb(nd.left_bb, lb);
        write_bb(nd.right_bb, rb);
        if (t.parent >= 0) (&nodes_out[t.parent].left)[t.child] = idx;
        SbvhTask tr{std::move(r), t.depth + 1, idx, 1};
        SbvhTask tl{std::move(l), t.depth + 1, idx, 0};
        stack.push_back(std::move(tr));
        stack.push_back(std::move(tl));
        l = std::vector<Ref>();
        r = std::vector<Ref>();
    }
    return 0;
}

}  // namespace
}  // namespace imbart

using namespace imbart;

extern "C" int imbart_build_mesh_node2_ex(const float* vertices, int n_vertices, int vertex_stride,
                                          const int* indices, int n_tris, int tri_offset, int leaf_size,
                                          float split_budget, imbart_node2* nodes_out, int nodes_cap, int* n_nodes,
                                          imbart_vec4* tris_out, int tris_cap, int* n_tri_vec4) {
    if (!vertices || !indices || !nodes_out || !tris_out || !n_nodes || !n_tri_vec4 ||
        n_tris <= 0 || vertex_stride < 3 || leaf_size < 1 || !(split_budget >= 0.0f)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_build_mesh_node2: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    std::vector<Prim> prims(n_tris);
    for (int t = 0; t < n_tris; ++t) {
        Prim& p = prims[t];
        p.box.reset();
        for (int k = 0; k < 3; ++k) {
            const int vi = indices[4 * t + k];
            if (vi < 0 || vi >= n_vertices) {
                set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_build_mesh_node2: vertex index out of range");
                return IMBART_ERR_INVALID_ARGUMENT;
            }
            p.box.grow(vertices + (size_t)vi * vertex_stride);
        }
        // Centroid of the vertices, as in fast_bvh_builder.h:36.
        for (int a = 0; a < 3; ++a) {
            const float* v0 = vertices + (size_t)indices[4 * t + 0] * vertex_stride;
            const float* v1 = vertices + (size_t)indices[4 * t + 1] * vertex_stride;
            const float* v2 = vertices + (size_t)indices[4 * t + 2] * vertex_stride;
            p.c[a] = (1.0f / 3.0f) * (v0[a] + v1[a] + v2[a]);
        }
    }
    auto emit_leaf = [&](const std::vector<int>& refs, int* code) -> int {
        if (*n_tri_vec4 + 3 * (int)refs.size() > tris_cap) return IMBART_ERR_LIMIT;
        *code = ~(*n_tri_vec4);
        for (int r : refs) {
            imbart_vec4* v = tris_out + *n_tri_vec4;
            for (int k = 0; k < 3; ++k) {
                const float* p = vertices + (size_t)indices[4 * r + k] * vertex_stride;
                v[k].x = p[0]; v[k].y = p[1]; v[k].z = p[2]; v[k].w = 0.0f;
            }
            v[1].w = bits_float(r + tri_offset);
            *n_tri_vec4 += 3;
        }
        tris_out[*n_tri_vec4 - 1].w = bits_float((int)0x80000000);
        return 0;
    };
    int err;
    if (split_budget > 0.0f) {
        // References allowed: the budget, and what the output buffers can hold (one node per
        // reference at most, three Vec4 per referenced triangle).
        std::vector<Tri3> tris(n_tris);
        for (int t = 0; t < n_tris; ++t)
            for (int k = 0; k < 3; ++k)
                for (int a = 0; a < 3; ++a) tris[t].v[k][a] = vertices[(size_t)indices[4 * t + k] * vertex_stride + a];
        long long max_refs = (long long)(n_tris * (1.0 + (double)split_budget));
        max_refs = std::min<long long>(max_refs, (tris_cap - (long long)*n_tri_vec4) / 3);
        max_refs = std::min<long long>(max_refs, nodes_cap - (long long)*n_nodes - 1);
        err = build_sbvh(tris, leaf_size, 4, 1.0f, max_refs, nodes_out, nodes_cap, n_nodes, emit_leaf);
    } else {
        // Traversal-cost factor 1.0 as the reference GPU mesh adapter (gpu_adapter.cpp:49-56).
        err = build_generic(prims, leaf_size, 4, 1.0f, nodes_out, nodes_cap, n_nodes, emit_leaf);
    }
    if (err) set_error(err, "imbart_build_mesh_node2: output capacity too small");
    return err;
}

extern "C" int imbart_build_mesh_node2(const float* vertices, int n_vertices, int vertex_stride,
                                       const int* indices, int n_tris, int tri_offset, int leaf_size,
                                       imbart_node2* nodes_out, int nodes_cap, int* n_nodes,
                                       imbart_vec4* tris_out, int tris_cap, int* n_tri_vec4) {
    return imbart_build_mesh_node2_ex(vertices, n_vertices, vertex_stride, indices, n_tris, tri_offset, leaf_size,
                                      0.0f, nodes_out, nodes_cap, n_nodes, tris_out, tris_cap, n_tri_vec4);
}

extern "C" int imbart_build_top_node2(const float* boxes, const float* inv_mats, const int* mesh_roots,
                                      int n_instances, imbart_node2* nodes_out, int nodes_cap, int* n_nodes,
                                      imbart_instance_node* inst_out) {
    if (!boxes || !inv_mats || !mesh_roots || !nodes_out || !n_nodes || !inst_out || n_instances <= 0) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_build_top_node2: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    std::vector<Prim> prims(n_instances);
    for (int i = 0; i < n_instances; ++i) {
        Prim& p = prims[i];
        for (int a = 0; a < 3; ++a) {
            p.box.lo[a] = boxes[6 * i + a];
            p.box.hi[a] = boxes[6 * i + 3 + a];
            p.c[a] = (p.box.lo[a] + p.box.hi[a]) * 0.5f;
        }
    }
    int n_written = 0;
    auto emit_leaf = [&](const std::vector<int>& refs, int* code) -> int {
        *code = ~n_written;
        for (int r : refs) {
            imbart_instance_node& in = inst_out[n_written++];
            std::memcpy(in.transf, inv_mats + 12 * (size_t)r, sizeof(in.transf));
            in.id = r;
            in.next = mesh_roots[r];
            in.pad[0] = 0; in.pad[1] = 0;
        }
        inst_out[n_written - 1].pad[0] = -1;
        inst_out[n_written - 1].pad[1] = -1;
        return 0;
    };
    // One instance per leaf and traversal-cost factor 0.5 as the reference top-level adapter
    // (gpu_adapter.cpp:188-197, leaf threshold 1 at :183).
    const int err = build_generic(prims, 1, 1, 0.5f, nodes_out, nodes_cap, n_nodes, emit_leaf);
    if (err) set_error(err, "imbart_build_top_node2: output capacity too small");
    return err;
}
