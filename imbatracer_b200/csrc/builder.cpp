// Binned-SAH BVH builder that writes the reference GPU two-wide layout.
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

}  // namespace
}  // namespace imbart

using namespace imbart;

extern "C" int imbart_build_mesh_node2(const float* vertices, int n_vertices, int vertex_stride,
                                       const int* indices, int n_tris, int tri_offset, int leaf_size,
                                       imbart_node2* nodes_out, int nodes_cap, int* n_nodes,
                                       imbart_vec4* tris_out, int tris_cap, int* n_tri_vec4) {
    if (!vertices || !indices || !nodes_out || !tris_out || !n_nodes || !n_tri_vec4 ||
        n_tris <= 0 || vertex_stride < 3 || leaf_size < 1) {
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
    // Traversal-cost factor 1.0 as the reference GPU mesh adapter (gpu_adapter.cpp:49-56).
    const int err = build_generic(prims, leaf_size, 4, 1.0f, nodes_out, nodes_cap, n_nodes, emit_leaf);
    if (err) set_error(err, "imbart_build_mesh_node2: output capacity too small");
    return err;
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
