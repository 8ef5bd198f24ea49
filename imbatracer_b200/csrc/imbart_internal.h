// Internal layouts of libimbart shared by the host-side builders/converters and the
// sm_100a kernels. Nothing here is part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/imbart.h"

namespace imbart {

// ---------------------------------------------------------------------------------------
// Compressed 8-wide BVH node, 80 bytes = 5 x 16 B, read with five 128-bit loads.
//
//   q0: px, py, pz (float grid origin), w = ex | ey << 8 | ez << 16 | imask << 24
//       (ex/ey/ez: signed 8-bit exponents, child box coordinate = p + q * 2^e;
//        imask bit s: slot s holds an internal child)
//   q1: child_base, prim_base, meta[0..3], meta[4..7]
//       internal child in slot s -> node child_base + popc(imask & ((1 << s) - 1))
//       leaf child in slot s     -> meta[s] = count << 5 | offset: primitives
//                                   [prim_base + offset, prim_base + offset + count)
//       empty slot               -> meta[s] = 0 and an inverted box
//   q2: qlo_x[0..7] (bytes 0-7), qhi_x[0..7] (bytes 8-15)
//   q3: qlo_y, qhi_y      q4: qlo_z, qhi_z
//
// Child slots are assigned at build time so that slot s holds the child lying towards
// (s&1 ? +x : -x, s&2 ? +y : -y, s&4 ? +z : -z); a ray with direction octant `oct` (bit set
// for a negative component) visits hit children in ascending order of (slot ^ oct),
// which approximates front-to-back order without sorting.
// ---------------------------------------------------------------------------------------
struct alignas(16) WideNode {
    float px, py, pz;
    uint8_t ex, ey, ez, imask;
    uint32_t child_base;
    uint32_t prim_base;
    uint8_t meta[8];
    uint8_t qlo_x[8], qhi_x[8];
    uint8_t qlo_y[8], qhi_y[8];
    uint8_t qlo_z[8], qhi_z[8];
};
static_assert(sizeof(WideNode) == 80, "WideNode must be 80 bytes");

// Triangle record, 48 bytes: v0.xyz + global tri id (int bits) in v0.w, v1.xyz, v2.xyz.
struct alignas(16) WideTri {
    float v0[3]; int32_t id;
    float v1[3]; int32_t pad0;
    float v2[3]; int32_t pad1;
};
static_assert(sizeof(WideTri) == 48, "WideTri must be 48 bytes");

// Instance record, 64 bytes: rows of the 3x4 world-to-object matrix, instance id and the
// wide index of the instanced mesh's root node.
struct alignas(16) WideInst {
    float m[12];
    int32_t id;
    int32_t root;
    int32_t pad[2];
};
static_assert(sizeof(WideInst) == 64, "WideInst must be 64 bytes");

// Per-ray root words (the traversal's per-ray roots) with this bit set name the mesh tree of a
// scene whose top level is one identity instance of id 0: the ray starts in that tree with the
// instance entry's transform by the identity. Node indices stay below 2^30.
constexpr int kDirectRootBit = 1 << 30;

// World-to-object rows exactly (1 0 0 0 / 0 1 0 0 / 0 0 1 0) (convert.cpp).
bool identity_instance(const WideInst& in);

// Host-side result of converting a reference layout.
struct HostWideScene {
    std::vector<WideNode> nodes;
    std::vector<WideTri> tris;
    std::vector<WideInst> insts;
    int root = 0;          // wide index of the top-level root
    int top_nodes = 0;     // number of top-level wide nodes
    int node_width = 8;    // children per node: 8, or 4 (slots 0..3 of the same record)
    bool masked = false;
    std::vector<int> indices;
    std::vector<imbart_vec2> texcoords;
    std::vector<imbart_mask_desc> masks;
    std::vector<uint8_t> mask_buffer;
};

// Converters (convert.cpp). Return empty string on success, else an error message.
// node_width: 8 or 4; -1 takes the process setting (current_node_width).
std::string convert_node2(int root, const imbart_node2* nodes, int n_nodes,
                          const imbart_instance_node* insts, int n_insts,
                          const imbart_vec4* tris, int n_tri_vec4, HostWideScene& out, int node_width = -1);
std::string convert_node4(int root, const imbart_node4* nodes, int n_nodes,
                          const imbart_instance_node* insts, int n_insts,
                          const imbart_vec4* tris, int n_tri_vec4, HostWideScene& out, int node_width = -1);
// Node width of the scenes converted from now on: IMBART_NODE_WIDTH or imbart_set_node_width.
int current_node_width();
// Decides whether the masks are all opaque and copies them when they are not.
void attach_masks(HostWideScene& out, const int* indices, int n_indices,
                  const imbart_vec2* texcoords, int n_texcoords,
                  const imbart_mask_desc* masks, int n_masks,
                  const char* mask_buffer, int mask_buffer_size);

// Thread-local error reporting (error.cpp).
void set_error(int code, const std::string& msg);

// Kernel launch accounting (error.cpp): every launch site adds its launches.
void note_launches(int n);
long long launches_total();

// Stream-ordered traversal launch used by the wavefront integrators (trace.cu). `stream` is
// a cudaStream_t; rays are imbart_ray records, hits imbart_hit records.
// `roots` (optional): per-ray root node for batches over several scenes of one pool;
// `count_ptr` (optional): device-resident ray count, `count` being its upper bound.
// `work` (optional): the persistent kernel's (next, done) counter pair, zeroed, owned by the
// caller (a launch inside a CUDA graph keeps its own); otherwise one of the device's ring.
int launch_trace_internal(const imbart_scene* scene, const void* rays, void* hits, float* v_out, int count,
                          int flags, void* stream, unsigned long long* stats, const int* roots = nullptr,
                          const int* count_ptr = nullptr, int* work = nullptr);

// Adds one traversal launch (as launch_trace_internal with count_ptr and work) to `graph`
// after `deps`, under the configuration in force; `count` > 0.
int add_trace_node(cudaGraph_t graph, const cudaGraphNode_t* deps, int n_deps, cudaGraphNode_t* node,
                   const imbart_scene* scene, const void* rays, void* hits, int count, int flags,
                   const int* count_ptr, int* work);

// The traversal configuration in force (variant, refill, postpone, any-hit variant and refill,
// coherent variant and refill, triangle batches of the three classes): a launch recorded in a
// graph is stale once it changes.
void trace_config_snapshot(int out[10]);
// Persistent traversal launches on `s` use this share (0.05..1) of the resident block slots,
// leaving the rest of the SMs to concurrent work on other streams.
void scene_set_grid_share(imbart_scene* s, float share);

// Every scene value a traversal launch takes into its parameters (array pointers, root,
// masks, device): two launches with equal keys and arguments are the same launch.
void scene_launch_key(const imbart_scene* s, unsigned long long out[12]);

// Device arrays of a built photon grid (hashgrid.cu): photons in bucket order (float4 xyz +
// index bits), inclusive bucket ends, the 10 grid parameters; false before the first build.
bool hashgrid_device_view(const imbart_hashgrid* g, const void** sorted, const int** cell_ends, const float** params,
                          int* table, int* n);

// Uploads a converted scene into arrays of its own (the path of imbart_scene_from_node2).
imbart_scene* upload_wide_scene(const HostWideScene& h, int device);

// A scene whose node, triangle and instance arrays are all `pool`, indexed in units of their
// own record sizes (WideNode, WideTri, WideInst); the pool stays owned by the caller.
imbart_scene* scene_pool_view(int device, const void* pool, size_t pool_bytes);
void scene_pool_view_destroy(imbart_scene* s);
// Root used by launches without a per-ray root array (single-scene work on the pool).
// The view's top-level root, and the mesh root and instance id of a top level that is one
// identity instance (direct_root -1: none).
void scene_pool_view_set_root(imbart_scene* s, int root, int direct_root = -1, int direct_inst = -1);

// A scene over device arrays built on the GPU; the scene takes ownership (cudaFree on
// destroy). NULL on error (the arrays are then still the caller's).
imbart_scene* scene_adopt_device_arrays(int device, WideNode* nodes, int64_t n_nodes, int64_t top_nodes,
                                        WideTri* tris, int64_t n_tris, WideInst* insts, int64_t n_insts, int root);

// imbart_estimate_pixel_size with the scratch buffers of a VCM context (kept between calls,
// so that repeated estimates allocate nothing once the context has grown to the image size).
int vcm_estimate_pixel_size(imbart_vcm* v, const imbart_scene* scene, const imbart_camera* cam, float* pixel_size,
                            void* stream);

inline int float_bits(float f) { union { float f; int i; } u; u.f = f; return u.i; }
inline float bits_float(int i) { union { float f; int i; } u; u.i = i; return u.f; }

}  // namespace imbart
