/*
 * imbart.h — C ABI of libimbart, the B200 (sm_100a) wavefront hot path of imbatracer.
 *
 * Two groups of entry points live here:
 *
 *  1. The four traversal symbols the reference links against (AnyDSL/traversal, which
 *     the reference includes from outside its tree, src/imbatracer/core/traversal_interface.h:4-10).
 *     They keep the reference's signatures and semantics exactly; see the comment on each.
 *     The matching drop-in headers for the reference's `namespace traversal_gpu { #include
 *     <traversal_gpu.h> }` pattern are include/traversal_gpu.h and include/traversal_cpu.h.
 *
 *  2. The extended imbart_* API: explicit scene preparation, asynchronous stream-ordered
 *     tracing of device buffers, the photon hash grid and error reporting.
 *
 * All functions are plain C: pointers and sizes, no C++ or torch types. Every pointer is
 * owned by the caller. Functions never abort or trap: failures set a thread-local error
 * readable through imbart_last_error() / imbart_last_error_string().
 */
#ifndef IMBART_H
#define IMBART_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------ */
/* Types of the reference boundary (byte layouts shared with include/traversal_*.h)      */
/* ------------------------------------------------------------------------------------ */

/* Vec4/Vec2 as used for triangles and texture coordinates (ray_queue.h:47-50). */
typedef struct { float x, y, z, w; } imbart_vec4;
typedef struct { float x, y; } imbart_vec2;

/* Ray: origin with tmin in org.w, direction with tmax in dir.w (camera.h:61-64, pt.cpp:37-41). 32 B. */
typedef struct { imbart_vec4 org; imbart_vec4 dir; } imbart_ray;

/* Hit: tri_id is the global triangle id (-1 = miss, ray_queue.h:168), inst_id the instance
 * index, tmax the hit distance and u the barycentric weight of the triangle's second vertex
 * (integrator.h:72-94, common.h:52-54). 16 B. */
typedef struct { int tri_id; int inst_id; float tmax; float u; } imbart_hit;

/* Two-wide BVH node written by the reference GPU adapter (gpu_adapter.cpp:84-101).
 * left/right >= 0: node index; < 0: ~(index of the first Vec4 of a triangle run in `tris`)
 * for bottom-level nodes, ~(index of the first instance node of a run) for top-level nodes.
 * A root that is a single leaf is wrapped in a parent whose right child is 0x76543210
 * (gpu_adapter.cpp:14-31). 64 B. */
typedef struct { float lo_x, hi_x, lo_y, hi_y, lo_z, hi_z; } imbart_bbox;
typedef struct { imbart_bbox left_bb; imbart_bbox right_bb; int left; int right; int pad[2]; } imbart_node2;

/* Four-wide SoA BVH node written by the reference CPU adapter (cpu_adapter.cpp:79-101).
 * children[j] > 0: node index; 0: empty slot; < 0: ~(index of the first Vec4 of a run of
 * 13-Vec4 triangle packets, closed by an all-0x80000000 sentinel Vec4). 112 B. */
typedef struct {
    float min_x[4], max_x[4], min_y[4], max_y[4], min_z[4], max_z[4];
    int children[4];
} imbart_node4;

/* Instance node (cpu_adapter.cpp:346-365, gpu_adapter.cpp:255-276): the instance's
 * inverse transform as a row-major 3x4 matrix, the instance id, the node index of the
 * instanced mesh's BVH root, and pad[0] == -1 on the last node of a leaf run. 64 B. */
typedef struct { float transf[12]; int id; int next; int pad[2]; } imbart_instance_node;

/* Transparency mask descriptor (mask.h:9-20): a width x height byte image at `offset` in
 * the mask buffer, selected by the material id stored in indices[4*tri+3]. */
typedef struct { int width; int height; int offset; } imbart_mask_desc;

/* ------------------------------------------------------------------------------------ */
/* 1. Drop-in traversal entry points                                                      */
/* ------------------------------------------------------------------------------------ */
/*
 * Closest hit over the two-level instanced BVH for `count` rays (replaces
 * traversal_gpu::intersect_gpu_masked_instanced, called at ray_queue.h:279-290).
 * Every pointer is a DEVICE pointer allocated by the caller. `count` is the queue size
 * rounded up to a multiple of 64 (ray_queue.h:60,273); padding rays (zeroed, ray_queue.h:74)
 * produce misses. The reference layout is converted to the compressed 8-wide layout on the
 * first call for a given `nodes` buffer and cached; imbart_invalidate_scenes() drops the
 * cache after the caller rewrites the buffers. Returns after the hits are written
 * (the caller copies them back right away, ray_queue.h:292).
 * Triangles hit at the same t are resolved to the smallest (inst_id, tri_id).
 */
void intersect_gpu_masked_instanced(int root, imbart_node2* nodes, imbart_instance_node* instances,
                                    imbart_vec4* tris, imbart_ray* rays, imbart_hit* hits,
                                    int* indices, imbart_vec2* texcoords, imbart_mask_desc* masks,
                                    char* mask_buffer, int count);

/* Any hit within [tmin, tmax] (replaces traversal_gpu::occluded_gpu_masked_instanced,
 * ray_queue.h:329-340). hits[i].tri_id >= 0 when ray i is occluded, -1 otherwise
 * (consumer: integrator.h:57). Same pointer conventions as above. */
void occluded_gpu_masked_instanced(int root, imbart_node2* nodes, imbart_instance_node* instances,
                                   imbart_vec4* tris, imbart_ray* rays, imbart_hit* hits,
                                   int* indices, imbart_vec2* texcoords, imbart_mask_desc* masks,
                                   char* mask_buffer, int count);

/* Host-buffer forms with the reference CPU layout (replace traversal_cpu::intersect_cpu_masked_instanced
 * and occluded_cpu_masked_instanced, ray_queue.h:254-265 and 304-315). All pointers are HOST
 * pointers; the scene is converted once and kept resident on the GPU, rays are copied to the
 * device and hits back inside the call. The B200 does the traversal: there is no CPU path. */
void intersect_cpu_masked_instanced(int root, imbart_node4* nodes, imbart_instance_node* instances,
                                    imbart_vec4* tris, imbart_ray* rays, imbart_hit* hits,
                                    int* indices, imbart_vec2* texcoords, imbart_mask_desc* masks,
                                    char* mask_buffer, int count);
void occluded_cpu_masked_instanced(int root, imbart_node4* nodes, imbart_instance_node* instances,
                                   imbart_vec4* tris, imbart_ray* rays, imbart_hit* hits,
                                   int* indices, imbart_vec2* texcoords, imbart_mask_desc* masks,
                                   char* mask_buffer, int count);

/* Drops every scene the drop-in entry points converted and cached. Call after rewriting
 * node, triangle or instance buffers in place (Scene::upload_top_level_accel, scene.cpp:167-188). */
void imbart_invalidate_scenes(void);

/* ------------------------------------------------------------------------------------ */
/* 2. Extended API                                                                         */
/* ------------------------------------------------------------------------------------ */

/* Error codes. */
enum {
    IMBART_OK = 0,
    IMBART_ERR_INVALID_ARGUMENT = 1,
    IMBART_ERR_CUDA = 2,
    IMBART_ERR_OUT_OF_MEMORY = 3,
    IMBART_ERR_BAD_SCENE = 4,
    IMBART_ERR_STACK_OVERFLOW = 5,
    IMBART_ERR_LIMIT = 6,
    IMBART_ERR_TIMEOUT = 7
};

/* Last error of the calling thread (0 = none) and its message; imbart_clear_error resets it. */
int imbart_last_error(void);
const char* imbart_last_error_string(void);
void imbart_clear_error(void);
/* Library version string. */
const char* imbart_version(void);

/* An opaque prepared scene: the compressed 8-wide BVH resident on one GPU. */
typedef struct imbart_scene imbart_scene;

/* Flags for scene preparation. */
enum { IMBART_SCENE_MASKED = 1 };

/* Prepares a scene from HOST arrays in the reference GPU (two-wide) layout.
 * n_nodes/n_tri_vec4/n_instances bound the arrays (for validation; the tree is walked from
 * `root`). indices/texcoords/masks/mask_buffer are only read when masks other than the
 * default opaque one are present (any mask with width*height > 1 or a zero texel).
 * Returns NULL on error. */
imbart_scene* imbart_scene_from_node2(int root, const imbart_node2* nodes, int n_nodes,
                                      const imbart_instance_node* instances, int n_instances,
                                      const imbart_vec4* tris, int n_tri_vec4,
                                      const int* indices, int n_indices,
                                      const imbart_vec2* texcoords, int n_texcoords,
                                      const imbart_mask_desc* masks, int n_masks,
                                      const char* mask_buffer, int mask_buffer_size,
                                      int device);

/* Same from HOST arrays in the reference CPU (four-wide, 13-Vec4 packet) layout. Vertices are
 * rebuilt as v1 = v0 - e1 and v2 = v0 + e2 from the packet's edges (cpu_adapter.cpp:129-201). */
imbart_scene* imbart_scene_from_node4(int root, const imbart_node4* nodes, int n_nodes,
                                      const imbart_instance_node* instances, int n_instances,
                                      const imbart_vec4* tris, int n_tri_vec4,
                                      const int* indices, int n_indices,
                                      const imbart_vec2* texcoords, int n_texcoords,
                                      const imbart_mask_desc* masks, int n_masks,
                                      const char* mask_buffer, int mask_buffer_size,
                                      int device);

void imbart_scene_destroy(imbart_scene* scene);

/* Node width of the scenes converted from the reference layouts from now on (process-wide):
 * 8 (the default), or 4, which fills slots 0..3 of the same 80 B record in x/y-quadrant order
 * and traverses with a 4-slot kernel. IMBART_NODE_WIDTH in the environment sets the initial
 * value. Hits never depend on the width; speed does (imbart_trace_autotune measures the
 * kernel shapes of one prepared scene, so comparing widths means preparing the scene once per
 * width). Scenes built on the device (imbart_scene_build_gpu) and loaded from .bvh files are
 * always 8-wide. Returns 0 or IMBART_ERR_INVALID_ARGUMENT. */
int imbart_set_node_width(int width);
int imbart_get_node_width(void);

/* Host-only conversion of the two-wide layout into the wide layout, without a GPU (for
 * inspection, byte accounting and tests), at the current node width. Writes up to the given
 * capacities and returns the required sizes in counts[0..3] = {wide nodes, triangles,
 * instances, root}. Call with zero capacities to query the sizes. Returns 0 or an error code. */
int imbart_wide_from_node2(int root, const imbart_node2* nodes, int n_nodes,
                           const imbart_instance_node* instances, int n_instances,
                           const imbart_vec4* tris, int n_tri_vec4,
                           void* nodes_out, int nodes_cap, void* tris_out, int tris_cap,
                           void* insts_out, int insts_cap, int* counts);

/* Sizes of a prepared scene. */
typedef struct {
    int64_t wide_nodes;        /* 80 B compressed 8-wide nodes (top and bottom level) */
    int64_t top_nodes;         /* of which top level */
    int64_t triangles;         /* 48 B triangle records (SBVH duplicates counted) */
    int64_t instances;         /* 64 B instance records */
    int64_t device_bytes;      /* total device memory held */
    int32_t root;              /* wide index of the top-level root */
    int32_t masked;            /* 1 when the alpha-mask test is active */
    int32_t node_width;        /* children per node: 8, or 4 */
    int32_t reserved;
} imbart_scene_info;
int imbart_scene_get_info(const imbart_scene* scene, imbart_scene_info* out);

/* Device pointers of the prepared scene's arrays (for measurement and tests):
 * nodes (80 B records), tris (3 float4 per triangle), instances (4 float4 per instance). */
int imbart_scene_get_device_arrays(const imbart_scene* scene, const void** nodes,
                                   const void** tris, const void** instances);

/* Trace flags. IMBART_TRACE_COHERENT (with closest hit) marks coherent rays, such as camera
 * rays in pixel order: they run with their own kernel configuration (see
 * imbart_set_trace_class). Hits never depend on the flags. */
enum { IMBART_TRACE_CLOSEST = 0, IMBART_TRACE_ANY = 1, IMBART_TRACE_COHERENT = 2 };

/* Traces `count` rays from DEVICE buffers, stream-ordered on `stream` (a cudaStream_t,
 * NULL = legacy default stream). Returns 0 or an error code; does not synchronize. */
int imbart_trace(const imbart_scene* scene, const imbart_ray* rays, imbart_hit* hits,
                 int count, int flags, void* stream);

/* Like imbart_trace, and also writes the barycentric weight of the third vertex per ray
 * to `v_out` (device, may be NULL) — the reference recomputes it (integrator.h:89-94). */
int imbart_trace_uv(const imbart_scene* scene, const imbart_ray* rays, imbart_hit* hits,
                    float* v_out, int count, int flags, void* stream);

/* Traces from HOST buffers (pinned or pageable): copies rays in, traces, copies hits out,
 * and synchronizes `stream`. */
int imbart_trace_host(const imbart_scene* scene, const imbart_ray* rays_host, imbart_hit* hits_host,
                      int count, int flags, void* stream);

/* Statistics variant of imbart_trace: same hits, and adds the numbers of 8-wide nodes
 * fetched, triangles tested and instances entered to stats[0..2] (DEVICE, 3 x uint64).
 * Used to compute the algorithmic bytes of a launch. */
int imbart_trace_stats(const imbart_scene* scene, const imbart_ray* rays, imbart_hit* hits, int count,
                       int flags, unsigned long long* stats, void* stream);

/* Number of rays that ran out of traversal stack (reported as misses) since the scene was
 * prepared; -1 on error. Synchronous. */
int imbart_scene_error_count(const imbart_scene* scene);

/* Number of kernel launches issued by this process so far (for launch accounting). */
int64_t imbart_kernel_launch_count(void);

/* Process-wide traversal kernel configuration (the tuning knobs of the autotuner):
 * variant 0 = one ray per thread; 1..10 = persistent warps (1: 128 threads x 4 blocks/SM,
 * 16-entry shared stack; 2: 128 x 6, 12; 3: 256 x 2, 16; 4: 256 x 3, 12; 5: 64 x 8, 16;
 * 6: 256 x 4, 8; 7: 128 x 7, 10; 8: 256 x 4, 12; 9: 256 x 4, 16; 10: 128 x 8, 12); refill_lanes (1..32): a warp fetches new rays once this
 * many lanes are idle; postpone_lanes (0..32): triangle tests are postponed while fewer than
 * postpone_lanes/32 of the live lanes would test together (0 = never).
 * imbart_set_trace_config sets the variant of both query types; imbart_set_trace_variant_any
 * then overrides the any-hit one. Defaults: closest 4, any-hit 6, refill 24, postpone 0
 * (environment: IMBART_TRACE_VARIANT, _VARIANT_ANY, _REFILL, _POSTPONE). */
int imbart_set_trace_config(int variant, int refill_lanes, int postpone_lanes);
int imbart_set_trace_variant_any(int variant);
int imbart_get_trace_config(int* variant, int* refill_lanes, int* postpone_lanes);
int imbart_get_trace_variant_any(void);

/* The configuration of one query class: flags IMBART_TRACE_CLOSEST (incoherent closest hit),
 * IMBART_TRACE_ANY, or IMBART_TRACE_CLOSEST | IMBART_TRACE_COHERENT. variant 1..17 (threads
 * per block x blocks per SM x shared stack entries of the persistent kernel; 1..10 test
 * triangles per lane, 11..17 with the cooperative triangle phase; 0: one ray per thread),
 * refill_lanes: idle lanes a warp waits for before it fetches new rays. */
int imbart_set_trace_class(int flags, int variant, int refill_lanes);
int imbart_get_trace_class(int flags, int* variant, int* refill_lanes);

/* Triangle batch of a query class (per-lane persistent shapes 1..10): the triangles a lane
 * tests per loop trip before the warp's lanes with node work take their next node step; 0 =
 * the whole leaf group at once. 0..24, default 0 (IMBART_TRACE_TRI_BATCH). The cooperative
 * shapes ignore it. Hits do not depend on it. */
int imbart_set_trace_tri_batch(int flags, int tri_batch);
int imbart_get_trace_tri_batch(int flags);

/* Autotuner: times every persistent-kernel configuration of the query class of `flags`
 * (variants 1..17 x refill 4, 8, 16, 24, 32, then triangle batches 0..4 of a per-lane best; one
 * warm-up and three timed launches each, CUDA events on `stream`) on `count` DEVICE rays,
 * keeps the fastest as the class's configuration and reports it with the time of the
 * configuration it replaced. Hits are written to `hits`.
 * Run it on rays like those the class will trace (camera rays, bounce rays, shadow rays). */
typedef struct {
    int variant;
    int refill;
    float ms;          /* per launch, the chosen configuration */
    float default_ms;  /* per launch, the configuration before tuning */
    int tri_batch;     /* the chosen triangle batch (imbart_set_trace_tri_batch) */
} imbart_trace_tuning;
int imbart_trace_autotune(const imbart_scene* scene, const imbart_ray* rays, imbart_hit* hits, int count, int flags,
                          void* stream, imbart_trace_tuning* out);

/* ------------------------------------------------------------------------------------ */
/* Photon hash grid (replaces HashGrid::build / HashGrid::query, rangesearch.h:25-129,     */
/* used by LightVertices::build / get_merge, light_vertices.h:70-100)                      */
/* ------------------------------------------------------------------------------------ */

typedef struct imbart_hashgrid imbart_hashgrid;

/* Creates an empty grid whose buffers live on `device`. NULL on error. */
imbart_hashgrid* imbart_hashgrid_create(int device);
void imbart_hashgrid_destroy(imbart_hashgrid* grid);

/* Builds the grid over n photon positions (DEVICE pointer; photon i's xyz at
 * positions + i * stride floats, stride >= 3). cell size = radius * cell_factor (the reference
 * uses 2, rangesearch.h:29); table_size buckets (<= 0: 2 * n, the reference's choice,
 * rangesearch.h:26). Stream-ordered; device buffers grow as needed and are kept. */
int imbart_hashgrid_build(imbart_hashgrid* grid, const float* positions, int stride, int n, float radius,
                          float cell_factor, int table_size, void* stream);

/* k-capped radius queries for nq positions (DEVICE, 3 packed floats each), 1 <= k <= 64.
 * out_ids (nq*k) receives the indices (build order) of the photons within the radius, at most
 * the k nearest, ordered by (squared distance, index) and padded with -1; out_counts (nq) the
 * count; out_d2 (nq*k, may be NULL) the squared distances. A bucket reached twice through the
 * 8 neighbour cells is scanned twice, as in the reference (rangesearch.h:94-104). Grids built
 * with 1 <= cell_factor < 2 are queried over every cell within the radius instead (each
 * bucket once); cell_factor < 1 is refused. */
int imbart_hashgrid_query(const imbart_hashgrid* grid, const float* queries, int nq, int k, int* out_ids,
                          int* out_counts, float* out_d2, void* stream);

/* The same build and queries on HOST arrays, for HashGrid::build / HashGrid::query callers
 * that hold their photons in host memory (as the reference's LightVertices does,
 * light_vertices.h:70-100): the library copies positions in and results out through its own
 * staging buffers and returns when done. Queries may run concurrently from several host
 * threads (each thread has its own staging buffers and stream); a build must not overlap
 * queries of the same grid. */
int imbart_hashgrid_build_host(imbart_hashgrid* grid, const float* positions, int stride, int n, float radius,
                               float cell_factor, int table_size);
int imbart_hashgrid_query_host(const imbart_hashgrid* grid, const float* queries, int nq, int k, int* out_ids,
                               int* out_counts, float* out_d2);

/* Grid parameters after a build (synchronous): params10 = {lo xyz, hi xyz, radius, radius^2,
 * cell size, 1 / cell size}, photon count and table size. */
int imbart_hashgrid_get_params(const imbart_hashgrid* grid, float* params10, int* n, int* table_size);

/* Device arrays of the built grid: photons in bucket order (float4: xyz + index bits) and
 * the inclusive bucket ends (table_size ints). */
int imbart_hashgrid_get_arrays(const imbart_hashgrid* grid, const void** sorted, const int** cell_ends);

/* Hash-grid build that allocates nothing (no counterpart in the reference). For callers that
 * must not allocate device memory: a server admitting work against a fixed HBM budget, where
 * cudaMalloc/cudaFree would also synchronize the device and stall other requests' streams,
 * or a host that hands out only device buffers from its own arena. Same result as
 * imbart_hashgrid_build, written to caller-owned DEVICE outputs: sorted_out (n float4: xyz +
 * photon index bits, in bucket order), cell_ends_out (table_size inclusive bucket ends) and
 * params_out (10 floats: lo xyz, hi xyz, radius, radius^2, cell size, 1/cell size). The build's
 * scratch is one static device array of about 12 MiB, held by every GPU that loads the library
 * until the process exits; it bounds n to 1,048,576 photons and table_size (<= 0: 2n) to
 * 2,097,152 buckets — larger requests return IMBART_ERR_LIMIT without launching anything.
 * The first call on a device looks the array's address up for that device
 * (cudaGetSymbolAddress with the device current). With CUDA's lazy module loading (the
 * default) that first call is also when the driver loads the module and reserves the array,
 * which can synchronize the device: make one call per device at start-up (n = 0 is enough),
 * before admitting work and before any stream capture. All calls share the one array: calls
 * that overlap on the GPU (different streams, no ordering between them) race and must be
 * serialized by the caller. A launch error pending on the calling thread is cleared on entry;
 * when the call fails after its first launch (IMBART_ERR_CUDA), the outputs are undefined.
 * Stream-ordered. */
int imbart_hashgrid_build_noalloc(const float* positions, int stride, int n, float radius, float cell_factor,
                                  int table_size, void* sorted_out, int* cell_ends_out, float* params_out,
                                  void* stream);

/* ------------------------------------------------------------------------------------ */
/* Sample generation and wavefront path tracing                                            */
/* ------------------------------------------------------------------------------------ */

/* Camera matrices of PerspectiveCamera::move (camera.h:27-56) for a camera at `pos` looking
 * along `dir` with `up`, horizontal field of view `fov` degrees, a width x height raster and
 * `aspect` (1 in the reference): raster_to_world and world_to_raster (16 floats row-major,
 * either output may be NULL except raster_to_world) and the image-plane distance. Host only. */
int imbart_camera_setup(const float* pos, const float* dir, const float* up, float fov, float width,
                        float height, float aspect, float* raster_to_world, float* world_to_raster,
                        float* img_plane_dist);

/* Camera samples first..first+count-1 of a width x height frame with `spp` samples per
 * pixel: the reference's PixelRayGen seeding (ray_gen.h:49-72, sample index = global index
 * into the frame) and the path tracer's pixel jitter (pt.cpp:168-177). DEVICE outputs: rays,
 * pixel ids, sample ids (may be NULL) and the 64-bit RNG state after the jitter draws. */
int imbart_camera_rays(const float* raster_to_world, const float* cam_pos, int width, int height, int spp,
                       unsigned long long seed_base, long long first, int count, imbart_ray* rays,
                       int* pixel_ids, int* sample_ids, unsigned long long* rng_states, void* stream);

/* Shading data of a scene, resident on one GPU: global vertex arrays (positions, normals,
 * texture coordinates), per global triangle {v0, v1, v2, material} and geometric normal,
 * per instance the 3x4 world-to-object matrix, materials (kind: 0 Lambertian, 1 mirror,
 * 2 glass, 3 glossy Cook-Torrance+Lambert, 4 Phong+Lambert, 5 emissive; 16 parameters:
 * colour[3], specular[3], exponent, eta, kappa, emission[3], unused[4]), triangle lights
 * (12 floats: p0, p1, p2, intensity; world space) and an optional constant environment
 * colour (light 0 when present). bsphere = scene bounding sphere {centre, radius, 1/r^2}. */
typedef struct imbart_shading imbart_shading;
imbart_shading* imbart_shading_create(int device, const float* vertices, int n_vertices, const float* normals,
                                      const float* texcoords, const int* tris, const float* geom_normals,
                                      int n_tris, const float* inst_inv, int n_inst, const int* mat_kind,
                                      const float* mat_params, int n_mats, const float* tri_lights,
                                      int n_tri_lights, const float* env_color, const float* bsphere);
/* Makes the environment light an image (EnvMap / EnvLight, light.h:361-544): texture
 * `texture` of the shading data (latitude-longitude, rgba) times `intensity`, looked up at
 * the texel the reference's EnvMap reads (no filtering; directions sampled uniformly over
 * the map, as the reference does). Adds the environment as light 0 when the scene had none. */
int imbart_shading_set_env_map(imbart_shading* shading, int texture, float intensity);
void imbart_shading_destroy(imbart_shading* shading);

/* imbart_shading_create with every light kind of the reference and textures.
 * Lights (12 floats each, after the environment in the light list), light_kinds[i] (NULL: all
 * triangles): 0 triangle {p0, p1, p2, intensity} (TriangleLight, light.h:94-190);
 * 1 directional {direction of travel (normalized), 6 unused, intensity} (DirectionalLight,
 * :192-237); 2 point {position, 6 unused, intensity} (PointLight, :239-290); 3 spot {position,
 * axis (normalized), half-angle in radians, 2 unused, intensity} (SpotLight, :292-355).
 * Textures (TextureSampler, texture_sampler.h:18-46): tex_dims[2t] = width, [2t+1] = height,
 * tex_pixels = the textures' rgba texels back to back, rows bottom-up as the reference indexes
 * them (texel (x, y) at y * width + x). Material params[12] = diffuse texture of a Lambertian,
 * glossy or Phong material, params[13] = bump map of any material (Material::bump,
 * materials.h:32-53); negative = none. */
imbart_shading* imbart_shading_create_ex(int device, const float* vertices, int n_vertices, const float* normals,
                                         const float* texcoords, const int* tris, const float* geom_normals,
                                         int n_tris, const float* inst_inv, int n_inst, const int* mat_kind,
                                         const float* mat_params, int n_mats, const int* light_kinds,
                                         const float* lights, int n_lights, const float* env_color,
                                         const float* bsphere, const int* tex_dims, const float* tex_pixels,
                                         int n_textures);

/* Wavefront path-tracing context (device queues, grown on demand). */
typedef struct imbart_pt_context imbart_pt_context;
imbart_pt_context* imbart_pt_create(int device);
void imbart_pt_destroy(imbart_pt_context* ctx);

/* Renders one frame of the path tracer (PathTracer, pt.cpp) into `image` (DEVICE,
 * width*height*3 floats, accumulated: contributions are added). max_path_len as in the
 * reference (path vertices incl. camera and light; a path continues while bounces + 1 <
 * max_path_len); Russian roulette from bounce `rr_start` on (0 = the reference). At most
 * max_paths_in_flight paths (<= 0: 16M) are in flight; larger frames run in consecutive
 * sample ranges with unchanged seeding. stats (host, may be NULL): closest-hit rays, shadow
 * rays, wavefronts. By default the bounce loop of a sample range runs as a CUDA graph (built
 * on the first call, rebuilt when a launch parameter other than the camera or the seed
 * changes, replayed once per range; kernels read their queue sizes on the device): the call
 * then returns without synchronizing, unless stats are asked for (one synchronization at the
 * end). With graphs off (imbart_pt_set_graphs) or a profile set, the loop is driven from the
 * host and synchronizes `stream` once per wavefront. */
int imbart_pt_render(imbart_pt_context* ctx, const imbart_scene* scene, const imbart_shading* shading,
                     const float* raster_to_world, const float* cam_pos, int width, int height, int spp,
                     int max_path_len, int rr_start, unsigned long long seed_base, float* image,
                     long long max_paths_in_flight, long long* stats, void* stream);

/* The samples [first_sample, first_sample + n_samples) of the same frame (sample indices 0 ..
 * width*height*spp - 1, seeded as in the whole frame): disjoint ranges rendered into images
 * that are then summed give the whole frame's image (up to the order of float additions), so
 * one frame can be split across devices (imbatracer_b200.distributed.render_frame_split).
 * imbart_pt_render is the range [0, width*height*spp). */
int imbart_pt_render_range(imbart_pt_context* ctx, const imbart_scene* scene, const imbart_shading* shading,
                           const float* raster_to_world, const float* cam_pos, int width, int height, int spp,
                           int max_path_len, int rr_start, unsigned long long seed_base, float* image,
                           long long max_paths_in_flight, long long first_sample, long long n_samples,
                           long long* stats, void* stream);

/* Measurement of the traversal launches inside imbart_pt_render (for roofline reporting). */
typedef struct {
    int events;                 /* in: time every traversal launch with CUDA events on the stream */
    int work;                   /* in: run the statistics variant (counts nodes/triangles/instances) */
    double closest_ms;          /* out: summed closest-hit launch time */
    double shadow_ms;           /* out: summed any-hit launch time */
    long long closest_launches; /* out */
    long long shadow_launches;  /* out */
    long long closest_rays;     /* out */
    long long shadow_rays;      /* out */
    unsigned long long closest_work[3]; /* out: nodes, triangles, instances (work != 0) */
    unsigned long long shadow_work[3];
} imbart_pt_profile;

/* Makes the following imbart_pt_render calls of `ctx` fill `profile` (NULL: stop). */
int imbart_pt_set_profile(imbart_pt_context* ctx, imbart_pt_profile* profile);

/* How imbart_pt_render runs its bounce loop: 0 driven from the host (one synchronization per
 * wavefront), 1 a CUDA graph (one chain of launches), 2 a CUDA graph whose shadow-ray work
 * runs on a branch beside the next bounce's closest-hit launch, -1 the environment's choice
 * (IMBART_PT_GRAPH, default 2). */
int imbart_pt_set_graphs(imbart_pt_context* ctx, int enable);

/* The queue order of RayQueue::sort_by_material (ray_queue.h:211-244) as a permutation:
 * perm (DEVICE, n ints) lists the indices of keys (DEVICE, n bytes; keys above 7 count as 7)
 * grouped by key in increasing key order, stably (indices increasing within a key). The path tracer, the
 * VCM passes and the server group every wavefront this way before shading (key = material
 * kind of the hit, 6 = miss, 7 = finished light-path slot). Stream-ordered. */
int imbart_group_by_key(const unsigned char* keys, int n, int* perm, void* stream);

/* ------------------------------------------------------------------------------------ */
/* VCM family: VCM, BPT, PPM, LT and the VCM path tracer (VCMIntegrator<algo>, vcm.cpp)    */
/* ------------------------------------------------------------------------------------ */

/* A PerspectiveCamera (camera.h:12-113): both raster matrices (row-major), position,
 * normalized view direction, image-plane distance and the raster size. */
typedef struct {
    float raster_to_world[16];
    float world_to_raster[16];
    float pos[3];
    float dir[3];
    float img_plane_dist;
    int width, height;
} imbart_camera;

/* PerspectiveCamera(width, height, fov).move(pos, dir, up) on the host. */
int imbart_camera_make(const float* pos, const float* dir, const float* up, float fov, int width, int height,
                       imbart_camera* out);

/* Integrator::estimate_pixel_size (integrator.cpp:14-70): the mean distance between the hit
 * points of rays through neighbouring raster corners of every 8th pixel (1 when nothing is
 * hit). The photon radius of the VCM family is this times its radius factor. Synchronous. */
int imbart_estimate_pixel_size(const imbart_scene* scene, const imbart_camera* camera, float* pixel_size,
                               void* stream);

#define IMBART_VCM 0      /* vertex connection and merging */
#define IMBART_BPT 1      /* bidirectional path tracing (no merging) */
#define IMBART_PPM 2      /* progressive photon mapping (camera paths sample only specular lobes) */
#define IMBART_LT 3       /* light tracing (light paths connected to the camera only) */
#define IMBART_VCM_PT 4   /* path tracing inside the VCM integrator (no light paths) */

/* The reference's UserSettings that drive VCMIntegrator (cmd_line.h:40-58). */
typedef struct {
    int algorithm;            /* IMBART_VCM .. IMBART_VCM_PT */
    int spp;                  /* camera samples per pixel per iteration (concurrent_spp) */
    int max_path_len;         /* vertices per path (camera path + light path for connections) */
    int light_path_count;     /* light paths per iteration */
    int num_connections;      /* light vertices each camera vertex connects to */
    int num_knn;              /* photons per merge (1..64) */
    int light_tile_size;      /* paths per light tile (the reference: tile_size^2); 0: one tile per light */
    float base_radius;        /* photon radius of iteration 1 (pixel size * radius factor) */
    unsigned long long light_seed, light_seed_step;  /* light tile t is seeded from light_seed + t * step */
    unsigned long long camera_seed;                  /* seed_base of the camera samples */
    /* Photon-grid schedule (zero = the reference's): the radius of iteration i is
     * base_radius * i^-radius_exponent (0: the reference's (1 - 0.75) / 2 = 1/8, vcm.cpp:27-38),
     * the grid's cells are grid_cell_factor radii wide (0: 2, rangesearch.h:27-30; at least 1)
     * and it has grid_table_size buckets (0: twice the photons, rangesearch.h:26,33-34). */
    float radius_exponent;
    float grid_cell_factor;
    int grid_table_size;
} imbart_vcm_settings;

/* Context with device buffers (light-path slots, light-vertex cache, photon grid, queues). */
typedef struct imbart_vcm imbart_vcm;
imbart_vcm* imbart_vcm_create(int device);
void imbart_vcm_destroy(imbart_vcm* vcm);

/* Iteration `iteration` (1-based): photon radius base / iteration^(0.5 * (1 - 0.75)) and the
 * MIS constants (vcm.cpp:25-46); out3 (may be NULL) = radius, eta_vc, eta_vm. Clears the cache. */
int imbart_vcm_begin_iteration(imbart_vcm* vcm, const imbart_vcm_settings* settings, int iteration, float* out3);

/* Light pass (trace_light_paths, vcm.cpp:64-104): traces light_path_count light paths, stores
 * their non-specular vertices in the cache (order: wavefront, then path), adds the camera
 * connections to `image` (DEVICE, width*height*3 floats) and builds the photon grid (VCM, PPM).
 * stats (host, may be NULL): closest rays, shadow rays, wavefronts. Synchronizes per wavefront. */
int imbart_vcm_light_pass(imbart_vcm* vcm, const imbart_scene* scene, const imbart_shading* shading,
                          const imbart_camera* camera, const imbart_vcm_settings* settings, float* image,
                          long long* stats, void* stream);

/* The light pass over paths [first_path, first_path + n_paths) of the iteration's
 * light_path_count (each path seeded by its global index, so the ranges of several GPUs
 * together trace exactly the single-GPU paths). The cache then holds this range's vertices
 * in (wavefront, path) order; wave_counts (HOST, may be NULL) receives the vertices each
 * wavefront added, at most wave_cap entries. With the ranges' caches concatenated wavefront
 * by wavefront in range order, imbart_vcm_load_light_vertices restores the single-GPU
 * cache. */
int imbart_vcm_light_pass_range(imbart_vcm* vcm, const imbart_scene* scene, const imbart_shading* shading,
                                const imbart_camera* camera, const imbart_vcm_settings* settings, int first_path,
                                int n_paths, float* image, int* wave_counts, int wave_cap, long long* stats,
                                void* stream);

/* Camera pass (trace_camera_paths, vcm.cpp:106-130, 322-611) against the current cache. */
int imbart_vcm_camera_pass(imbart_vcm* vcm, const imbart_scene* scene, const imbart_shading* shading,
                           const imbart_camera* camera, const imbart_vcm_settings* settings, float* image,
                           long long max_paths_in_flight, long long* stats, void* stream);

/* The camera pass over camera samples [first_sample, first_sample + n_samples) of the
 * width * height * spp samples (sample index as in PixelRayGen: pixel-major per spp). */
int imbart_vcm_camera_pass_range(imbart_vcm* vcm, const imbart_scene* scene, const imbart_shading* shading,
                                 const imbart_camera* camera, const imbart_vcm_settings* settings,
                                 long long first_sample, long long n_samples, float* image,
                                 long long max_paths_in_flight, long long* stats, void* stream);

/* begin_iteration + light pass + camera pass into `image` (accumulated). */
int imbart_vcm_render(imbart_vcm* vcm, const imbart_scene* scene, const imbart_shading* shading,
                      const imbart_camera* camera, const imbart_vcm_settings* settings, int iteration, float* image,
                      long long max_paths_in_flight, long long* stats, void* stream);

/* The light-vertex cache: DEVICE pointer to `count` vertices of 28 floats (pos, material |
 * out_dir, path_length | normal, dVC | geom_normal, dVCM | u_tangent, dVM | v_tangent, uv.x |
 * throughput, uv.y; material and path_length as int32 bits). Valid until the next pass. */
int imbart_vcm_light_vertices(imbart_vcm* vcm, const float** vertices, int* count);

/* Copies up to `capacity` cache vertices to HOST memory (synchronous); returns the number
 * copied, or the cache's vertex count when capacity is 0, or -(error code). */
int imbart_vcm_copy_light_vertices(imbart_vcm* vcm, float* host_out, int capacity);

/* Replaces the cache with `count` vertices in that format (HOST or DEVICE) and rebuilds the
 * photon grid (VCM, PPM) for the current iteration's radius: camera passes can then run
 * against a cache produced elsewhere (the reference's, a previous frame's). */
int imbart_vcm_load_light_vertices(imbart_vcm* vcm, const imbart_vcm_settings* settings, const float* vertices,
                                   int count, void* stream);

/* ------------------------------------------------------------------------------------ */
/* Request serving (no counterpart in the reference, which renders one frame per process)  */
/* ------------------------------------------------------------------------------------ */

/* A server owns one GPU and a worker thread. Render requests (path-traced frames) and ray
 * batches (closest-hit / any-hit queries) are submitted from any host thread and complete
 * asynchronously.
 *
 * IMBART_SERVE_BATCHED: continuous batching. All resident scenes live in one device pool of
 * `hbm_budget_bytes` (scene data and render accumulation images); a scene is uploaded when a
 * request needs it, and when the pool is full the least recently used scene without
 * outstanding requests is evicted. Every wavefront merges the paths of all admitted render
 * requests (new camera samples are admitted between wavefronts, max-min fair across requests,
 * up to `max_paths_in_flight` paths) and the rays of all admitted ray batches, and runs one
 * closest-hit launch, one shading launch and one any-hit launch over all of them, whatever
 * their scenes.
 * IMBART_SERVE_PLAIN: the same requests one at a time in arrival order through the
 * single-request entry points (imbart_pt_render, imbart_trace) on scenes uploaded once each
 * (the budget is not applied). This is the baseline the batched mode is measured against.
 *
 * A request renders the same image in both modes and alone or in any mix (up to the order
 * of float additions into its image); a ray batch returns the same hits as imbart_trace. */
#define IMBART_SERVE_BATCHED 0
#define IMBART_SERVE_PLAIN 1

typedef struct imbart_server imbart_server;

/* Scene registration data: traversal arrays in the reference GPU layout (as
 * imbart_scene_from_node2, unmasked) and shading arrays (as imbart_shading_create). All
 * HOST pointers; the server keeps its own copies. */
typedef struct {
    int root;
    const imbart_node2* nodes; int n_nodes;
    const imbart_instance_node* instances; int n_instances;
    const imbart_vec4* tris; int n_tri_vec4;
    const float* vertices; int n_vertices;
    const float* normals; const float* texcoords;
    const int* mesh_tris; const float* geom_normals; int n_mesh_tris;
    const float* inst_inv; int n_inst_inv;
    const int* mat_kind; const float* mat_params; int n_mats;
    const float* tri_lights; int n_tri_lights;
    const float* env_color;    /* NULL: no environment light */
    const float* bsphere;      /* NULL: zero */
    /* Optional, as in imbart_shading_create_ex: kinds of the n_tri_lights lights (NULL: all
     * triangles) and textures (n_textures = 0: none). */
    const int* light_kinds;
    const int* tex_dims;
    const float* tex_pixels;
    int n_textures;
    /* Optional: 1 + the texture holding an environment image (0: none) and its intensity,
     * as imbart_shading_set_env_map. */
    int env_map;
    float env_intensity;
} imbart_scene_source;

/* One path-traced frame (as imbart_pt_render with a fresh zeroed image). image_host: HOST
 * width*height*3 floats, written before the request completes. */
typedef struct {
    int scene;
    float raster_to_world[16];
    float cam_pos[3];
    int width, height, spp, max_path_len, rr_start;
    unsigned long long seed_base;
    float* image_host;
} imbart_render_request;

/* One VCM-family frame (VCM, BPT, PPM, LT, VCM-PT; VCMIntegrator::render, vcm.cpp:25-55, once
 * per iteration) into a fresh zeroed image: iterations 1 .. `iterations` of imbart_vcm_render,
 * so the photon radius shrinks as over one long render. Iteration i draws its light tiles
 * from settings.light_seed + (i - 1) * seed_step and its camera samples from
 * settings.camera_seed + (i - 1) * seed_step. settings.base_radius <= 0 selects
 * radius_factor times imbart_estimate_pixel_size of the camera (the reference's default:
 * radius factor 2). image_host: HOST width*height*3 floats, the sum over the iterations.
 * In batched mode the request is admitted like a render (scene resident, image in the
 * pool); its iterations then run on VCM lanes (host threads with their own CUDA streams and
 * VCM contexts; IMBART_SERVE_VCM_LANES, default 4), one iteration at a time and round robin
 * over the admitted VCM-family requests, concurrently with the merged wavefronts. */
typedef struct {
    int scene;
    imbart_camera camera;
    imbart_vcm_settings settings;
    float radius_factor;
    int iterations;
    unsigned long long seed_step;
    float* image_host;
} imbart_vcm_request;

/* Completion record. Times are milliseconds of the host steady clock since the server was
 * created: submission, admission (scene resident, memory granted) and completion (result in
 * the caller's buffer). */
typedef struct {
    int status;          /* 0 or an IMBART_ERR_* code */
    int kind;            /* 0 render, 1 ray batch, 2 VCM-family frame */
    double submit_ms, start_ms, done_ms;
} imbart_request_result;

typedef struct {
    long long submitted, completed, failed;
    long long waves;             /* merged wavefronts (batched) or per-request wavefronts (plain) */
    long long closest_rays, shadow_rays, batch_rays;
    long long scene_uploads, scene_evictions;
    long long pool_bytes, pool_used_bytes;
    long long kernel_launches;
} imbart_server_stats;

/* hbm_budget_bytes: device pool for scenes and images (batched mode; <= 0: 4 GiB);
 * max_paths_in_flight: paths per merged wavefront (<= 0: 4M); also the limit of ray-batch
 * rays per wavefront. NULL on error (imbart_last_error). */
imbart_server* imbart_server_create(int device, int mode, long long hbm_budget_bytes, long long max_paths_in_flight);
/* Waits for every submitted request, then stops the worker and frees the device memory. */
void imbart_server_destroy(imbart_server* server);
/* Registers a scene; returns its id (>= 0) or -(error code). Scenes are not uploaded until
 * a request needs them. */
int imbart_server_add_scene(imbart_server* server, const imbart_scene_source* source);

/* Registers a scene whose traversal arrays are built on the server's GPU from its meshes
 * and instances (imbart_scene_build_gpu: a fraction of a second where the host SBVH build
 * and conversion take seconds for millions of triangles) instead of taken from `source`,
 * whose traversal fields are then ignored (the shading fields are as for
 * imbart_server_add_scene). The built arrays are kept on the host like a converted scene's,
 * so the pool uploads and evicts the scene the same way. build_ms (may be NULL): wall time
 * of the build and its download. */
typedef struct imbart_mesh_desc imbart_mesh_desc;
typedef struct imbart_instance_desc imbart_instance_desc;
int imbart_server_add_scene_gpu_build(imbart_server* server, const imbart_scene_source* source,
                                      const imbart_mesh_desc* meshes, int n_meshes,
                                      const imbart_instance_desc* instances, int n_instances, float* build_ms);
/* Submits a request; returns a ticket (> 0) or -(error code). */
long long imbart_server_submit_render(imbart_server* server, const imbart_render_request* request);
long long imbart_server_submit_vcm(imbart_server* server, const imbart_vcm_request* request);
/* rays / hits: HOST (pageable or pinned) or DEVICE pointers of `count` records; flags
 * IMBART_TRACE_CLOSEST or IMBART_TRACE_ANY. */
long long imbart_server_submit_rays(imbart_server* server, int scene, const imbart_ray* rays, imbart_hit* hits,
                                    int count, int flags);
/* Blocks until the request completed; fills `result` (may be NULL) and forgets the ticket.
 * Returns the request's status (IMBART_ERR_INVALID_ARGUMENT for an unknown ticket). */
int imbart_server_wait(imbart_server* server, long long ticket, imbart_request_result* result);
/* Blocks until every request submitted so far completed. */
int imbart_server_drain(imbart_server* server);
int imbart_server_get_stats(imbart_server* server, imbart_server_stats* stats);

/* ------------------------------------------------------------------------------------ */
/* BVH construction (the builder side of the boundary)                                     */
/* ------------------------------------------------------------------------------------ */

/* Builds one mesh's bottom-level BVH with a binned SAH (32 bins, leaf threshold
 * `leaf_size`) and APPENDS it in the reference GPU two-wide layout: nodes to
 * `nodes_out` (capacity `nodes_cap`), triangle Vec4 triples (global id = tri_offset + local
 * id in v1.w, sentinel 0x80000000 in the last v2.w of each leaf) to `tris_out` (capacity
 * `tris_cap` Vec4s). `*n_nodes` / `*n_tri_vec4` are in/out fill counts. `vertices` are
 * xyz floats with stride `vertex_stride` floats, `indices` 4 ints per triangle
 * {i0, i1, i2, material} (mesh.h:103-114). Node indices written are absolute in nodes_out.
 * Returns 0 or an error code (IMBART_ERR_LIMIT when a capacity is too small). */
int imbart_build_mesh_node2(const float* vertices, int n_vertices, int vertex_stride,
                            const int* indices, int n_tris, int tri_offset, int leaf_size,
                            imbart_node2* nodes_out, int nodes_cap, int* n_nodes,
                            imbart_vec4* tris_out, int tris_cap, int* n_tri_vec4);

/* imbart_build_mesh_node2 with spatial splits (SBVH, Stich et al. 2009, as the reference's
 * SplitBvhBuilder offers, sbvh_builder.h:29-165): where the two children of the best object
 * split overlap, triangles may be split at a binned plane and referenced from both sides
 * (each with its box clipped to its side). split_budget bounds the extra references as a
 * fraction of n_tris (0: object splits only, the same tree as imbart_build_mesh_node2); the
 * output capacities bound them too. Hits are the same as over any other tree. */
int imbart_build_mesh_node2_ex(const float* vertices, int n_vertices, int vertex_stride,
                               const int* indices, int n_tris, int tri_offset, int leaf_size, float split_budget,
                               imbart_node2* nodes_out, int nodes_cap, int* n_nodes,
                               imbart_vec4* tris_out, int tris_cap, int* n_tri_vec4);

/* Builds the top-level BVH over instance boxes (binned SAH, one instance per leaf) and
 * APPENDS it in the reference two-wide layout at node index `*n_nodes` (the root is that
 * index), writing instance nodes to `inst_out` (`n_instances` of them). inv_mats are the
 * 3x4 row-major inverse transforms, mesh_roots[i] the BVH root node of instance i's mesh,
 * boxes the world-space instance boxes (6 floats: lo xyz, hi xyz). */
int imbart_build_top_node2(const float* boxes, const float* inv_mats, const int* mesh_roots,
                           int n_instances, imbart_node2* nodes_out, int nodes_cap, int* n_nodes,
                           imbart_instance_node* inst_out);

/* ------------------------------------------------------------------------------------ */
/* GPU scene build (no counterpart in the reference, which builds on the CPU with SBVH)    */
/* ------------------------------------------------------------------------------------ */

/* A triangle mesh: HOST arrays of n_vertices xyz floats and n_tris {v0, v1, v2, material}
 * ints; tri_offset is the global id of its first triangle (hits report tri_offset + local
 * index, as Scene::build_mesh_accels numbers triangles, scene.cpp:75-97). */
struct imbart_mesh_desc {
    const float* vertices; int n_vertices;
    const int* indices; int n_tris;
    int tri_offset;
};

/* An instance: row-major 3x4 object-to-world and world-to-object matrices, the mesh it
 * instances and the id its hits report. */
struct imbart_instance_desc {
    float obj_to_world[12];
    float world_to_obj[12];
    int mesh;
    int id;
};

/* Builds a scene entirely on the GPU (PLOC clustering over Morton-sorted primitives, a
 * surface-area leaf pass, a collapse into the compressed 8-wide layout) and returns it ready
 * for imbart_trace and the renderers, like imbart_scene_from_node2 (unmasked). One BVH per
 * mesh, a top-level BVH over the instances. Synchronizes `stream`; build_ms (may be NULL)
 * receives the wall time. NULL on error (imbart_last_error). */
imbart_scene* imbart_scene_build_gpu(const imbart_mesh_desc* meshes, int n_meshes,
                                     const imbart_instance_desc* instances, int n_instances, int device,
                                     void* stream, float* build_ms);

/* Refit (no counterpart in the reference, which rebuilds on the CPU): after a scene's mesh
 * vertices moved with the topology unchanged, rewrites its triangle records from the new
 * positions and recomputes every node box bottom-up — the meshes' BVHs, the instances' world
 * boxes, the top level — with the build's conservative quantization, so traversal finds the
 * closest hits of the moved triangles exactly (the tree may fit them less tightly than a
 * rebuild). vertices: DEVICE xyz floats (object space) of every mesh's vertices, n_vertices
 * of them; tri_vertices: DEVICE {v0, v1, v2, unused} per global triangle id, indexing
 * `vertices` (the layout of the shading data's triangles). For scenes with their own arrays
 * (imbart_scene_from_node2/4, imbart_scene_build_gpu), not views of a server's pool.
 * Synchronizes `stream`. */
int imbart_scene_refit(imbart_scene* scene, const float* vertices, long long n_vertices, const int* tri_vertices,
                       int n_tri_ids, void* stream);

/* ------------------------------------------------------------------------------------ */
/* Acceleration-structure cache files (.bvh), as the reference reads and writes them      */
/* (load_accel_gpu / load_accel_cpu / store_accel_gpu / store_accel_cpu,                   */
/* src/imbatracer/loaders/load_bvh.cpp:44-304; used by Scene::build_mesh_accels,          */
/* scene.cpp:37-70)                                                                       */
/* ------------------------------------------------------------------------------------ */

/* File: u32 magic 0x313F1A57, then blocks [u64 size][u32 type][u32 node_count][u32
 * prim_count][nodes][prim_count Vec4s], size counting the bytes after the size field.
 * Block type 1 holds two-wide GPU nodes (imbart_node2), type 2 four-wide CPU nodes
 * (imbart_node4); a file holds at most one of each. Every size is checked: a malformed or
 * truncated file returns IMBART_ERR_BAD_SCENE. */
#define IMBART_ACCEL_GPU 1
#define IMBART_ACCEL_CPU 2

/* Node and Vec4 counts of the block of `block_type`. Returns 0, -1 when the file is valid
 * but has no such block, or an error code. */
int imbart_accel_file_info(const char* path, int block_type, int* node_count, int* vec4_count);

/* Appends the file's two-wide block at nodes_out[*n_nodes] / tris_out[*n_tri_vec4] (both
 * in/out counts, as the builders), rebasing node and leaf links when other nodes precede it
 * and adding tri_id_offset to the triangle ids (v1.w), as load_accel_gpu does. The
 * single-leaf wrapper's 0x76543210 marker is kept as it is (the reference shifts it with
 * the node offset). The result goes to imbart_scene_from_node2 like a built BVH. */
int imbart_load_accel_node2(const char* path, int tri_id_offset, imbart_node2* nodes_out, int nodes_cap,
                            int* n_nodes, imbart_vec4* tris_out, int tris_cap, int* n_tri_vec4);

/* The four-wide block (load_accel_cpu): ids are the last Vec4 of each 13-Vec4 packet. */
int imbart_load_accel_node4(const char* path, int tri_id_offset, imbart_node4* nodes_out, int nodes_cap,
                            int* n_nodes, imbart_vec4* tris_out, int tris_cap, int* n_vec4);

/* Appends the mesh BVH nodes[node_offset, n_nodes) / tris[tris_offset, n_tri_vec4) to the
 * file as a block with links relative to the mesh and ids minus tri_id_offset
 * (store_accel_gpu); creates the file when it does not exist, refuses
 * (IMBART_ERR_INVALID_ARGUMENT) when it has a two-wide block already. */
int imbart_store_accel_node2(const char* path, const imbart_node2* nodes, int node_offset, int n_nodes,
                             const imbart_vec4* tris, int tris_offset, int n_tri_vec4, int tri_id_offset);

/* The four-wide block (store_accel_cpu). */
int imbart_store_accel_node4(const char* path, const imbart_node4* nodes, int node_offset, int n_nodes,
                             const imbart_vec4* tris, int tris_offset, int n_vec4, int tri_id_offset);

#ifdef __cplusplus
}
#endif

#endif /* IMBART_H */
