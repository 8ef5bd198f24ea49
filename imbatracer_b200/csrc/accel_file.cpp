// Reader and writer of the reference's acceleration-structure cache files (.bvh).
//
// The reference keeps one file per mesh and, when building a scene, loads the mesh's BVH
// from it or builds the BVH and appends it to the file (Scene::build_mesh_accels,
// src/imbatracer/render/scene.cpp:37-70; format in src/imbatracer/loaders/load_bvh.cpp).
// The format is kept as it is, so that files written by the reference load here and files
// written here load in the reference:
//
//   u32 magic 0x313F1A57, then blocks of
//   u64 size | u32 type (1: two-wide GPU nodes, 2: four-wide CPU nodes) |
//   u32 node_count | u32 prim_count | node_count nodes | prim_count Vec4s
//
// where size counts the bytes after the size field (type, counts, data). A file holds at
// most one block of each type. Node links in a block are relative to the mesh's first node
// and first Vec4; loading appends to arrays that already hold other meshes and rebases the
// links, storing makes them relative again (load_bvh.cpp:44-142 and 144-304). Unlike the
// reference, every size is checked against the file and the caller's capacities, and a
// malformed file is an error, not a crash.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "imbart_internal.h"

namespace imbart {
namespace {

constexpr uint32_t kMagic = 0x313F1A57u;
constexpr uint32_t kBlockGpu = 1;      // BlockType::BVH  (two-wide, traversal_gpu::Node)
constexpr uint32_t kBlockCpu = 2;      // BlockType::MBVH (four-wide, traversal_cpu::Node)
constexpr int kDummyRight = 0x76543210;
constexpr int kSentinel = (int)0x80000000;
constexpr int kPacketVec4 = 13;        // four-wide triangle packet: 12 coordinate Vec4s + 1 id Vec4

struct File {
    std::FILE* f = nullptr;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() { if (f) std::fclose(f); }
};

struct BlockInfo {
    uint32_t node_count = 0, prim_count = 0;
    long long data = 0;    // file offset of the first node
};

bool read_at(std::FILE* f, long long off, void* dst, size_t bytes) {
    return std::fseek(f, (long)off, SEEK_SET) == 0 && std::fread(dst, 1, bytes, f) == bytes;
}

long long file_size(std::FILE* f) {
    if (std::fseek(f, 0, SEEK_END) != 0) return -1;
    return (long long)std::ftell(f);
}

// 0: found; 1: the file is valid but has no block of `type`; an error code otherwise.
int find_block(std::FILE* f, uint32_t type, size_t node_bytes, BlockInfo* out) {
    const long long size = file_size(f);
    uint32_t magic = 0;
    if (size < 4 || !read_at(f, 0, &magic, 4) || magic != kMagic) return IMBART_ERR_BAD_SCENE;
    long long pos = 4;
    while (pos < size) {
        uint64_t bsize = 0;
        uint32_t btype = 0;
        if (pos + 12 > size || !read_at(f, pos, &bsize, 8) || !read_at(f, pos + 8, &btype, 4)) return IMBART_ERR_BAD_SCENE;
        if (bsize < 12 || (long long)bsize > size - pos - 8) return IMBART_ERR_BAD_SCENE;
        if (btype == type) {
            uint32_t counts[2];
            if (!read_at(f, pos + 12, counts, 8)) return IMBART_ERR_BAD_SCENE;
            const unsigned long long need = 12ull + node_bytes * counts[0] + 16ull * counts[1];
            if (need > bsize || counts[0] > (uint32_t)INT32_MAX || counts[1] > (uint32_t)INT32_MAX)
                return IMBART_ERR_BAD_SCENE;
            out->node_count = counts[0];
            out->prim_count = counts[1];
            out->data = pos + 20;
            return 0;
        }
        pos += 8 + (long long)bsize;
    }
    return 1;
}

int fail(int code, const std::string& what) {
    set_error(code, what);
    return code;
}

// Appends the block's nodes and Vec4s at *n_nodes / *n_vec4 (load_accel_gpu / _cpu).
template <typename Node, typename Rebase, typename Ids>
int load_block(const char* path, uint32_t type, const char* name, Node* nodes_out, int nodes_cap, int* n_nodes,
               imbart_vec4* tris_out, int tris_cap, int* n_vec4, Rebase rebase, Ids fix_ids) {
    if (!path || !nodes_out || !tris_out || !n_nodes || !n_vec4 || *n_nodes < 0 || *n_vec4 < 0 ||
        *n_nodes > nodes_cap || *n_vec4 > tris_cap)
        return fail(IMBART_ERR_INVALID_ARGUMENT, std::string(name) + ": invalid argument");
    File file(path, "rb");
    if (!file.f) return fail(IMBART_ERR_INVALID_ARGUMENT, std::string(name) + ": cannot open " + path);
    BlockInfo b;
    const int rc = find_block(file.f, type, sizeof(Node), &b);
    if (rc == 1) return fail(IMBART_ERR_BAD_SCENE, std::string(name) + ": no block of this type in " + path);
    if (rc) return fail(rc, std::string(name) + ": malformed file " + path);
    if ((long long)*n_nodes + b.node_count > nodes_cap || (long long)*n_vec4 + b.prim_count > tris_cap)
        return fail(IMBART_ERR_LIMIT, std::string(name) + ": output capacity too small");
    const int node_offset = *n_nodes, tris_offset = *n_vec4;
    if (!read_at(file.f, b.data, nodes_out + node_offset, sizeof(Node) * b.node_count) ||
        !read_at(file.f, b.data + (long long)sizeof(Node) * b.node_count, tris_out + tris_offset,
                 sizeof(imbart_vec4) * b.prim_count))
        return fail(IMBART_ERR_BAD_SCENE, std::string(name) + ": truncated file " + path);
    // Links are rebased only when other nodes precede the block, as the reference does.
    if (node_offset > 0)
        for (uint32_t i = 0; i < b.node_count; ++i) rebase(nodes_out[node_offset + i], node_offset, tris_offset);
    fix_ids(tris_out + tris_offset, (int)b.prim_count);
    *n_nodes = node_offset + (int)b.node_count;
    *n_vec4 = tris_offset + (int)b.prim_count;
    return 0;
}

// Appends a block (store_accel_gpu / _cpu): refused when the file already has one of this type.
template <typename Node, typename Relink, typename Ids>
int store_block(const char* path, uint32_t type, const char* name, const Node* nodes, int node_offset, int n_nodes,
                const imbart_vec4* tris, int tris_offset, int n_vec4, Relink relink, Ids unfix_ids) {
    if (!path || !nodes || !tris || node_offset < 0 || tris_offset < 0 || n_nodes < node_offset ||
        n_vec4 < tris_offset)
        return fail(IMBART_ERR_INVALID_ARGUMENT, std::string(name) + ": invalid argument");
    bool exists = false;
    {
        File in(path, "rb");
        if (in.f) {
            BlockInfo b;
            const int rc = find_block(in.f, type, sizeof(Node), &b);
            if (rc == 0) return fail(IMBART_ERR_INVALID_ARGUMENT, std::string(name) + ": the file has this block already");
            exists = rc == 1;
        }
    }
    std::vector<Node> nb(nodes + node_offset, nodes + n_nodes);
    if (node_offset > 0)
        for (Node& n : nb) relink(n, node_offset, tris_offset);
    std::vector<imbart_vec4> tb(tris + tris_offset, tris + n_vec4);
    unfix_ids(tb.data(), (int)tb.size());
    File out(path, exists ? "ab" : "wb");
    if (!out.f) return fail(IMBART_ERR_INVALID_ARGUMENT, std::string(name) + ": cannot write " + path);
    const uint32_t counts[2] = {(uint32_t)nb.size(), (uint32_t)tb.size()};
    const uint64_t bsize = 4 + 8 + sizeof(Node) * nb.size() + sizeof(imbart_vec4) * tb.size();
    bool good = true;
    if (!exists) good = std::fwrite(&kMagic, 4, 1, out.f) == 1;
    good = good && std::fwrite(&bsize, 8, 1, out.f) == 1 && std::fwrite(&type, 4, 1, out.f) == 1 &&
           std::fwrite(counts, 8, 1, out.f) == 1 &&
           (nb.empty() || std::fwrite(nb.data(), sizeof(Node), nb.size(), out.f) == nb.size()) &&
           (tb.empty() || std::fwrite(tb.data(), sizeof(imbart_vec4), tb.size(), out.f) == tb.size());
    if (!good) return fail(IMBART_ERR_INVALID_ARGUMENT, std::string(name) + ": write failed for " + path);
    return 0;
}

int fbits(float f) { int i; std::memcpy(&i, &f, 4); return i; }
float bitsf(int i) { float f; std::memcpy(&f, &i, 4); return f; }

// The single-leaf root wrapper of gpu_adapter.cpp:14-31: left is the leaf, the right box is
// (0, -0) on every axis and right is the 0x76543210 marker.
bool is_leaf_wrapper(const imbart_node2& n) {
    const imbart_bbox& b = n.right_bb;
    return n.left < 0 && fbits(b.lo_x) == 0 && fbits(b.lo_y) == 0 && fbits(b.lo_z) == 0 && fbits(b.hi_x) == kSentinel &&
           fbits(b.hi_y) == kSentinel && fbits(b.hi_z) == kSentinel;
}

void rebase_node2(imbart_node2& n, int node_offset, int tris_offset) {
    const bool wrapper = is_leaf_wrapper(n);
    n.left = n.left < 0 ? ~(~n.left + tris_offset) : n.left + node_offset;
    n.right = n.right < 0 ? ~(~n.right + tris_offset) : n.right + node_offset;
    // The reference adds the node offset to the marker too; a file read back at another
    // offset than it was written at would then point past the nodes. Keep the marker.
    if (wrapper) n.right = kDummyRight;
}

void relink_node2(imbart_node2& n, int node_offset, int tris_offset) {
    const bool wrapper = is_leaf_wrapper(n);
    n.left = n.left < 0 ? ~(~n.left - tris_offset) : n.left - node_offset;
    n.right = n.right < 0 ? ~(~n.right - tris_offset) : n.right - node_offset;
    if (wrapper) n.right = kDummyRight;
}

void rebase_node4(imbart_node4& n, int node_offset, int tris_offset) {
    for (int j = 0; j < 4; ++j) {
        if (n.children[j] > 0) n.children[j] += node_offset;
        else if (n.children[j] < 0) n.children[j] = ~(~n.children[j] + tris_offset);
    }
}

void relink_node4(imbart_node4& n, int node_offset, int tris_offset) {
    for (int j = 0; j < 4; ++j) {
        if (n.children[j] > 0) n.children[j] -= node_offset;
        else if (n.children[j] < 0) n.children[j] = ~(~n.children[j] - tris_offset);
    }
}

// Two-wide layout: the triangle id is v1.w of every 3-Vec4 record (gpu_adapter.cpp:129-141).
void shift_ids_node2(imbart_vec4* t, int n, int delta) {
    if (delta == 0) return;
    for (int i = 0; i + 2 < n; i += 3) t[i + 1].w = bitsf(fbits(t[i + 1].w) + delta);
}

// Four-wide layout: packets of 13 Vec4s whose last Vec4 holds four ids (0x80000000 for an
// empty lane), a run closed by an all-0x80000000 sentinel Vec4 (cpu_adapter.cpp:150-180).
void shift_ids_node4(imbart_vec4* t, int n, int delta) {
    if (delta == 0) return;
    auto shift = [delta](float& v) { if (fbits(v) != kSentinel) v = bitsf(fbits(v) + delta); };
    for (int i = 0; i + kPacketVec4 <= n;) {
        i += kPacketVec4;
        imbart_vec4& ids = t[i - 1];
        shift(ids.x); shift(ids.y); shift(ids.z); shift(ids.w);
        if (i < n && fbits(t[i].x) == kSentinel) ++i;
    }
}

}  // namespace
}  // namespace imbart

using namespace imbart;

extern "C" {

int imbart_accel_file_info(const char* path, int block_type, int* node_count, int* vec4_count) {
    if (!path || (block_type != (int)kBlockGpu && block_type != (int)kBlockCpu))
        return fail(IMBART_ERR_INVALID_ARGUMENT, "imbart_accel_file_info: invalid argument");
    File file(path, "rb");
    if (!file.f) return fail(IMBART_ERR_INVALID_ARGUMENT, std::string("imbart_accel_file_info: cannot open ") + path);
    BlockInfo b;
    const int rc = find_block(file.f, (uint32_t)block_type,
                              block_type == (int)kBlockGpu ? sizeof(imbart_node2) : sizeof(imbart_node4), &b);
    if (rc > 1) return fail(rc, std::string("imbart_accel_file_info: malformed file ") + path);
    if (node_count) *node_count = rc == 0 ? (int)b.node_count : 0;
    if (vec4_count) *vec4_count = rc == 0 ? (int)b.prim_count : 0;
    return rc == 0 ? 0 : -1;
}

int imbart_load_accel_node2(const char* path, int tri_id_offset, imbart_node2* nodes_out, int nodes_cap, int* n_nodes,
                            imbart_vec4* tris_out, int tris_cap, int* n_tri_vec4) {
    return load_block<imbart_node2>(path, kBlockGpu, "imbart_load_accel_node2", nodes_out, nodes_cap, n_nodes,
                                    tris_out, tris_cap, n_tri_vec4, rebase_node2,
                                    [&](imbart_vec4* t, int n) { shift_ids_node2(t, n, tri_id_offset); });
}

int imbart_load_accel_node4(const char* path, int tri_id_offset, imbart_node4* nodes_out, int nodes_cap, int* n_nodes,
                            imbart_vec4* tris_out, int tris_cap, int* n_vec4) {
    return load_block<imbart_node4>(path, kBlockCpu, "imbart_load_accel_node4", nodes_out, nodes_cap, n_nodes,
                                    tris_out, tris_cap, n_vec4, rebase_node4,
                                    [&](imbart_vec4* t, int n) { shift_ids_node4(t, n, tri_id_offset); });
}

int imbart_store_accel_node2(const char* path, const imbart_node2* nodes, int node_offset, int n_nodes,
                             const imbart_vec4* tris, int tris_offset, int n_tri_vec4, int tri_id_offset) {
    return store_block<imbart_node2>(path, kBlockGpu, "imbart_store_accel_node2", nodes, node_offset, n_nodes, tris,
                                     tris_offset, n_tri_vec4, relink_node2,
                                     [&](imbart_vec4* t, int n) { shift_ids_node2(t, n, -tri_id_offset); });
}

int imbart_store_accel_node4(const char* path, const imbart_node4* nodes, int node_offset, int n_nodes,
                             const imbart_vec4* tris, int tris_offset, int n_vec4, int tri_id_offset) {
    return store_block<imbart_node4>(path, kBlockCpu, "imbart_store_accel_node4", nodes, node_offset, n_nodes, tris,
                                     tris_offset, n_vec4, relink_node4,
                                     [&](imbart_vec4* t, int n) { shift_ids_node4(t, n, -tri_id_offset); });
}

}  // extern "C"
