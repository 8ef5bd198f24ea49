// Harness around the reference's own C++ (compiled in place from the reference tree into
// oracle/_ref/libref.so by oracle/ref/build_ref.py). TEST INFRASTRUCTURE ONLY: it runs the
// reference's RNG, camera, ray generation, HashGrid, BVH builders/adapters, Scene and
// integrators on the CPU to pin the oracle and to produce golden outputs. The traversal
// behind the reference's traversal_gpu entry points is the oracle's CPU restatement
// (oracle/traversal.c), since the reference's AnyDSL traversal library is not in its tree.
#include <fcntl.h>
#include <unistd.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "imbatracer/render/scene.h"
#include "imbatracer/core/adapter.h"
#include "imbatracer/loaders/loaders.h"
#include "imbatracer/rangesearch/rangesearch.h"
#include "imbatracer/render/integrators/pt.h"
#include "imbatracer/render/ray_gen/camera.h"
#include "imbatracer/render/ray_gen/ray_gen.h"
#include "imbatracer/render/ray_gen/tile_gen.h"
#include "imbatracer/render/random.h"
#include "imbatracer/render/scheduling/tile_scheduler.h"

uint64_t imbart_ref_seed_value = 0;
uint64_t imbart_ref_seed_step = 0;
int imbart_ref_tbb_threads = 1;

// The oracle's two-wide traversal (oracle/traversal.c).
extern "C" void oracle_trace_node2(int root, const void* nodes, const void* insts, const void* tris,
                                   const int* indices, const void* texcoords, const void* masks, int n_masks,
                                   const uint8_t* mask_buffer, const void* rays, void* hits, float* v_out,
                                   int count, int any, int threads);

namespace {
int g_masks_active = 0;
int g_n_masks = 0;
int g_trace_threads = 1;

// The alpha-mask test is active for scenes whose uploaded masks are not all the default
// opaque 1x1 descriptor (scenes read from files with map_d), as the reference's traversal
// applies them.
void use_scene_masks(const imba::Scene& scene) {
    const auto& td = scene.traversal_data_gpu();
    g_masks_active = 0;
    g_n_masks = (int)td.masks.size();
    // A host copy: under the device-memory shim (libref_imbart.so) the arrays are on the GPU.
    using Mask = typename std::decay<decltype(td.masks.data()[0])>::type;
    anydsl::Array<Mask> host(anydsl::Platform::Host, anydsl::Device(0), td.masks.size());
    anydsl::copy(td.masks, host, td.masks.size());
    for (int64_t i = 0; i < host.size(); ++i) {
        const auto& m = host.data()[i];
        if (m.width * m.height > 1) g_masks_active = 1;
    }
}
}

#ifndef IMBART_REF_TRAVERSAL_FROM_IMBART
// The reference's GPU entry points, served on the CPU by the oracle. (The build that links
// libimbart instead, libref_imbart.so, leaves them to libimbart.)
extern "C" void intersect_gpu_masked_instanced(int root, traversal_gpu::Node* nodes, traversal_gpu::InstanceNode* insts,
                                               traversal_gpu::Vec4* tris, traversal_gpu::Ray* rays,
                                               traversal_gpu::Hit* hits, int* indices, traversal_gpu::Vec2* texcoords,
                                               traversal_gpu::TransparencyMask* masks, char* mask_buffer, int count) {
    oracle_trace_node2(root, nodes, insts, tris, g_masks_active ? indices : nullptr, texcoords,
                       g_masks_active ? masks : nullptr, g_n_masks, (const uint8_t*)mask_buffer, rays, hits, nullptr,
                       count, 0, g_trace_threads);
}
extern "C" void occluded_gpu_masked_instanced(int root, traversal_gpu::Node* nodes, traversal_gpu::InstanceNode* insts,
                                              traversal_gpu::Vec4* tris, traversal_gpu::Ray* rays,
                                              traversal_gpu::Hit* hits, int* indices, traversal_gpu::Vec2* texcoords,
                                              traversal_gpu::TransparencyMask* masks, char* mask_buffer, int count) {
    oracle_trace_node2(root, nodes, insts, tris, g_masks_active ? indices : nullptr, texcoords,
                       g_masks_active ? masks : nullptr, g_n_masks, (const uint8_t*)mask_buffer, rays, hits, nullptr,
                       count, 1, g_trace_threads);
}
// The CPU-layout entry points are referenced by the reference's scheduler templates but
// never reached: the harness always selects the GPU traversal path.
extern "C" void intersect_cpu_masked_instanced(int, traversal_cpu::Node*, traversal_cpu::InstanceNode*,
                                               traversal_cpu::Vec4*, traversal_cpu::Ray*, traversal_cpu::Hit* hits,
                                               int*, traversal_cpu::Vec2*, traversal_cpu::TransparencyMask*, char*,
                                               int count) {
    for (int i = 0; i < count; ++i) hits[i].tri_id = -1;
}
extern "C" void occluded_cpu_masked_instanced(int, traversal_cpu::Node*, traversal_cpu::InstanceNode*,
                                              traversal_cpu::Vec4*, traversal_cpu::Ray*, traversal_cpu::Hit* hits,
                                              int*, traversal_cpu::Vec2*, traversal_cpu::TransparencyMask*, char*,
                                              int count) {
    for (int i = 0; i < count; ++i) hits[i].tri_id = -1;
}
#endif

using namespace imba;

namespace {

// Phong material for workloads that ask for one: a 50/50 mix of the reference's Phong and
// Lambertian BxDFs (brdfs.h:8-91), built like GlossyMaterial (materials.h:151-189).
class PhongMaterialRef : public Material {
public:
    PhongMaterialRef(float exponent, const rgb& spec, const rgb& diff, const TextureSampler* diff_sampler = nullptr,
                     const TextureSampler* bump = nullptr)
        : Material(bump), exponent_(exponent), spec_(spec), diff_(diff), diff_sampler_(diff_sampler) {}
    Material* duplicate() const override { return new PhongMaterialRef(exponent_, spec_, diff_, diff_sampler_, bump_); }
    BSDF* get_bsdf(const Intersection& isect, MemoryArena& arena, bool) const override {
        auto a = arena.alloc<Phong>(spec_, exponent_);
        auto b = arena.alloc<Lambertian>(diff_sampler_ ? diff_sampler_->sample(isect.uv) : diff_);
        auto brdf = arena.alloc<CombineBxDF>(a, b);
        return arena.alloc<BSDF>(isect, brdf, nullptr);
    }

private:
    float exponent_;
    rgb spec_, diff_;
    const TextureSampler* diff_sampler_;
};

// Options of the next ref_scene_create: the CPU (four-wide) layout too, and acceleration
// cache file names per mesh (empty: none), as Scene::build_mesh_accels takes them.
bool g_next_cpu_buffers = false;
std::vector<std::string> g_next_accel_files;

struct RefScene {
    RefScene() : scene(g_next_cpu_buffers, true) {}
    Scene scene;
    MaskBuffer masks;
    std::vector<int> mat_kind;
    std::vector<float> mat_params;
};

float3 f3(const float* p) { return float3(p[0], p[1], p[2]); }

}  // namespace

imba::Scene* ref_scene_of(void* h) { return &static_cast<RefScene*>(h)->scene; }

// An empty scene (GPU layout only) for the scene-file loader harness (ref_scene_io.cpp).
void* ref_scene_new_empty() { return new RefScene; }

extern "C" {

void imbart_ref_set_seed(uint64_t value, uint64_t step) {
    imbart_ref_seed_value = value;
    imbart_ref_seed_step = step;
}

void imbart_ref_set_threads(int tbb_threads, int trace_threads) {
    imbart_ref_tbb_threads = tbb_threads < 1 ? 1 : tbb_threads;
    g_trace_threads = trace_threads < 1 ? 1 : trace_threads;
}

// MWC64X draws (random.h:15-47).
void ref_rng_floats(uint64_t seed, int n, float* out) {
    RNG rng(seed);
    for (int i = 0; i < n; ++i) out[i] = rng.random_float();
}

void ref_rng_ints(uint64_t seed, int n, int lo, int hi, int* out) {
    RNG rng(seed);
    for (int i = 0; i < n; ++i) out[i] = rng.random_int(lo, hi);
}

// Camera samples of one frame through PixelRayGen::fill_queue (ray_gen.h:36-80) with the
// path tracer's pixel sampling (pt.cpp:168-177) and PerspectiveCamera (camera.h:27-65).
// Writes rays (8 floats), pixel ids, sample ids and the RNG state after sampling.
int ref_camera_rays(int w, int h, int spp, const float* pos, const float* dir, const float* up, float fov,
                    uint64_t seed_base, float* rays_out, int* pixel_ids, int* sample_ids, uint64_t* rng_states) {
    PerspectiveCamera cam((float)w, (float)h, fov);
    cam.move(f3(pos), f3(dir), f3(up));
    const int n = w * h * spp;
    RayQueue<PTState> q(n, false);
    PixelRayGen<PTState> gen(w, h, spp);
    gen.start_frame();
    imbart_ref_set_seed(seed_base, 0);
    gen.fill_queue(q, [&](int x, int y, ::Ray& ray_out, PTState& st) {
        const float sx = static_cast<float>(x) + st.rng.random_float();
        const float sy = static_cast<float>(y) + st.rng.random_float();
        ray_out = cam.generate_ray(sx, sy);
        st.throughput = rgb(1.0f);
        st.bounces = 0;
        st.last_specular = false;
    });
    if (q.size() != n) return -1;
    std::memcpy(rays_out, q.rays(), sizeof(float) * 8 * n);
    for (int i = 0; i < n; ++i) {
        pixel_ids[i] = q.states()[i].pixel_id;
        sample_ids[i] = q.states()[i].sample_id;
        std::memcpy(rng_states + i, &q.states()[i].rng, sizeof(uint64_t));
    }
    return n;
}

// HashGrid::build + query (rangesearch.h:25-129) over n photons; output ids are the photons'
// indices in the input, in the order the reference's query returns them.
struct RefPhotonIn {
    float3 p;
    int id;
    float3& position() { return p; }
    const float3& position() const { return p; }
};
struct RefPhoton {
    float3 position;
    int id;
    RefPhoton() {}
    RefPhoton(const RefPhotonIn& in) : position(in.p), id(in.id) {}
};

int ref_hashgrid_query(const float* pos, int n, float radius, const float* queries, int nq, int k, int* out_ids,
                       int* out_counts) {
    std::vector<RefPhotonIn> ph(n);
    for (int i = 0; i < n; ++i) { ph[i].p = float3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]); ph[i].id = i; }
    HashGrid<std::vector<RefPhotonIn>::iterator, RefPhoton> grid;
    grid.build(ph.begin(), ph.end(), radius);
    std::vector<const RefPhoton*> out(k);
    for (int q = 0; q < nq; ++q) {
        const float3 qp(queries[3 * q], queries[3 * q + 1], queries[3 * q + 2]);
        const int c = grid.query(qp, out, k);
        out_counts[q] = c;
        for (int j = 0; j < k; ++j) out_ids[(size_t)q * k + j] = j < c ? out[j]->id : -1;
    }
    return 0;
}

// Scene from arrays. Materials: kind per material (0 Lambert, 1 mirror, 2 glass, 3 glossy,
// 4 phong, 5 emissive) and 16 parameters each: color[3], specular[3], exponent, eta, kappa,
// emission[3]. Lights: 12 floats each (p0, p1, p2, intensity), world space. env: 3 floats or
// NULL (a constant environment as a 1x1 EnvMap, listed before the triangle lights as the
// reference's scene parser adds it).
void* ref_scene_create(int n_meshes, const int* mesh_nverts, const int* mesh_ntris, const float* verts,
                       const int* indices, const float* normals, const float* texcoords, const float* geom_normals,
                       int n_inst, const int* inst_mesh, const float* inst_mats, int n_mats, const int* mat_kind,
                       const float* mat_params, int n_lights, const float* lights, const float* env) {
    RefScene* rs = new RefScene;
    Scene& scene = rs->scene;
    size_t vo = 0, io = 0;
    for (int m = 0; m < n_meshes; ++m) {
        scene.meshes().emplace_back();
        Mesh& mesh = scene.meshes().back();
        mesh.add_attribute(Mesh::AttributeType::FLOAT2);
        mesh.add_attribute(Mesh::AttributeType::FLOAT3);
        mesh.add_attribute(Mesh::AttributeType::FLOAT3, Mesh::AttributeBinding::PER_FACE);
        mesh.set_index_count(4 * (size_t)mesh_ntris[m]);
        mesh.set_vertex_count(mesh_nverts[m]);
        for (int i = 0; i < 4 * mesh_ntris[m]; ++i) mesh.indices()[i] = (uint32_t)indices[io + i];
        auto tc = mesh.attribute<float2>(MeshAttributes::TEXCOORDS);
        auto nr = mesh.attribute<float3>(MeshAttributes::NORMALS);
        auto gn = mesh.attribute<float3>(MeshAttributes::GEOM_NORMALS);
        for (int v = 0; v < mesh_nverts[m]; ++v) {
            const size_t g = vo + v;
            mesh.vertices()[v] = float4(verts[3 * g], verts[3 * g + 1], verts[3 * g + 2], 1.0f);
            tc[v] = float2(texcoords[2 * g], texcoords[2 * g + 1]);
            nr[v] = float3(normals[3 * g], normals[3 * g + 1], normals[3 * g + 2]);
        }
        for (int t = 0; t < mesh_ntris[m]; ++t) {
            const size_t g = io / 4 + t;
            gn[t] = float3(geom_normals[3 * g], geom_normals[3 * g + 1], geom_normals[3 * g + 2]);
        }
        vo += mesh_nverts[m];
        io += 4 * (size_t)mesh_ntris[m];
        mesh.compute_bounding_box();
    }
    for (int i = 0; i < n_inst; ++i) {
        const float* a = inst_mats + 16 * i;
        float4x4 mat(float4(a[0], a[1], a[2], a[3]), float4(a[4], a[5], a[6], a[7]), float4(a[8], a[9], a[10], a[11]),
                     float4(a[12], a[13], a[14], a[15]));
        scene.instances().emplace_back(inst_mesh[i], mat);
    }
    if (env) {
        Image img(1, 1);
        img(0, 0) = float4(env[0], env[1], env[2], 1.0f);
        scene.set_env_map(new EnvMap(img, 1.0f, scene.bounding_sphere()));
        scene.lights().emplace_back(new EnvLight(scene.env_map(), scene.bounding_sphere()));
    }
    rs->mat_kind.assign(mat_kind, mat_kind + n_mats);
    rs->mat_params.assign(mat_params, mat_params + 16 * (size_t)n_mats);
    for (int m = 0; m < n_mats; ++m) {
        const float* p = mat_params + 16 * m;
        const rgb color(p[0], p[1], p[2]), spec(p[3], p[4], p[5]), emit(p[9], p[10], p[11]);
        Material* mat = nullptr;
        switch (mat_kind[m]) {
            case 1: mat = new MirrorMaterial(p[7], p[8], color); break;
            case 2: mat = new GlassMaterial(p[7], color, spec); break;
            case 3: mat = new GlossyMaterial(p[6], spec, color); break;
            case 4: mat = new PhongMaterialRef(p[6], spec, color); break;
            default: mat = new DiffuseMaterial(color); break;
        }
        scene.materials().emplace_back(mat);
        rs->masks.add_desc();
    }
    for (int l = 0; l < n_lights; ++l) {
        const float* p = lights + 12 * l;
        scene.lights().emplace_back(new TriangleLight(rgb(p[9], p[10], p[11]), f3(p), f3(p + 3), f3(p + 6)));
    }
    // Emitters of emissive materials: the area of the face in object space (build_scene.cpp:233).
    io = 0;
    for (int m = 0; m < n_meshes; ++m) {
        const Mesh& mesh = scene.meshes()[m];
        for (int t = 0; t < mesh_ntris[m]; ++t) {
            const int mat = indices[io + 4 * t + 3];
            if (mat_kind[mat] != 5) continue;
            const float* p = mat_params + 16 * mat;
            const Tri tri = mesh.triangle(t);
            scene.material(mat)->set_emitter(new AreaEmitter(rgb(p[9], p[10], p[11]), tri.area()));
        }
        io += 4 * (size_t)mesh_ntris[m];
    }
    std::vector<std::string> names(n_meshes, "");
    if ((int)g_next_accel_files.size() == n_meshes) names = g_next_accel_files;
    g_next_accel_files.clear();
    g_next_cpu_buffers = false;
    scene.build_mesh_accels(names);
    scene.build_top_level_accel();
    scene.compute_bounding_sphere();
    scene.upload_mesh_accels();
    scene.upload_top_level_accel();
    scene.upload_mask_buffer(rs->masks);
    return rs;
}

void ref_scene_destroy(void* h) { delete static_cast<RefScene*>(h); }

// Adds the reference's other light kinds after the scene's lights (kinds 1 directional,
// 2 point, 3 spot; 12 floats each, the layout of imbart_shading_create_ex) and textures
// (TextureSampler over rgba texels, texel (x, y) at y * width + x), then rebuilds the
// materials with a diffuse texture (mat_tex) or a bump map (mat_bump); -1 = none.
int ref_scene_extend(void* h, int n_lights, const int* kinds, const float* lights, int n_tex, const int* tex_dims,
                     const float* tex_pixels, const int* mat_tex, const int* mat_bump) {
    RefScene* rs = static_cast<RefScene*>(h);
    Scene& scene = rs->scene;
    for (int l = 0; l < n_lights; ++l) {
        const float* q = lights + 12 * l;
        const rgb intensity(q[9], q[10], q[11]);
        switch (kinds[l]) {
            case 1: scene.lights().emplace_back(new DirectionalLight(f3(q), intensity, scene.bounding_sphere())); break;
            case 2: scene.lights().emplace_back(new PointLight(f3(q), intensity)); break;
            case 3: scene.lights().emplace_back(new SpotLight(f3(q), f3(q + 3), q[6], intensity)); break;
            default: return -1;
        }
    }
    const int first_tex = (int)scene.textures().size();
    size_t off = 0;
    for (int t = 0; t < n_tex; ++t) {
        const int w = tex_dims[2 * t], ht = tex_dims[2 * t + 1];
        Image img(w, ht);
        for (int i = 0; i < w * ht; ++i) {
            const float* p = tex_pixels + 4 * (off + i);
            img.pixels()[i] = float4(p[0], p[1], p[2], p[3]);
        }
        off += (size_t)w * ht;
        scene.textures().emplace_back(new TextureSampler(std::move(img)));
    }
    for (int m = 0; mat_tex && mat_bump && m < (int)rs->mat_kind.size(); ++m) {
        if (mat_tex[m] < 0 && mat_bump[m] < 0) continue;
        const float* p = rs->mat_params.data() + 16 * m;
        const rgb color(p[0], p[1], p[2]), spec(p[3], p[4], p[5]);
        TextureSampler* tex = mat_tex[m] >= 0 ? scene.texture(first_tex + mat_tex[m]).get() : nullptr;
        TextureSampler* bump = mat_bump[m] >= 0 ? scene.texture(first_tex + mat_bump[m]).get() : nullptr;
        Material* mat = nullptr;
        switch (rs->mat_kind[m]) {
            case 1: mat = new MirrorMaterial(p[7], p[8], color, bump); break;
            case 2: mat = new GlassMaterial(p[7], color, spec, bump); break;
            case 3: mat = tex ? new GlossyMaterial(p[6], spec, tex, bump) : new GlossyMaterial(p[6], spec, color, bump); break;
            case 4: mat = new PhongMaterialRef(p[6], spec, color, tex, bump); break;
            case 5: return -2;   // emissive faces keep their plain material
            default: mat = tex ? new DiffuseMaterial(tex, bump) : new DiffuseMaterial(color, bump); break;
        }
        scene.materials()[m].reset(mat);
    }
    return 0;
}

// Samplers of the reference evaluated with a fresh RNG(seed). Several of them take two
// rng.random_float() calls as arguments of one call, whose evaluation order C++ leaves to
// the compiler; the values here show which draw went to which argument in this build.
void ref_probe_samplers(uint64_t seed, float* out) {
    {
        RNG rng(seed);
        Lambertian l(rgb(1.0f));
        float3 in;
        float pdf;
        l.sample(float3(0.0f, 0.0f, 1.0f), in, rng, pdf);   // sample_cos_hemisphere (bsdf.h:54-64)
        out[0] = in.x; out[1] = in.y; out[2] = in.z;
    }
    {
        RNG rng(seed);
        TriangleLight t(rgb(1.0f), float3(0, 0, 0), float3(1, 0, 0), float3(0, 1, 0));
        auto s = t.sample_direct(float3(0.2f, 0.2f, 1.0f), rng);   // sample_uniform_triangle (light.h:146)
        out[3] = s.dir.x; out[4] = s.dir.y; out[5] = s.dir.z;
    }
    {
        RNG rng(seed);
        FresnelConductor f(1.0f, 20.0f);
        CookTorrance ct(rgb(1.0f), &f, 20.0f);
        float3 in;
        float pdf;
        ct.sample(float3(0.3f, 0.1f, 0.9f), in, rng, pdf);   // sample_blinn_distribution (brdfs.h:177)
        out[6] = in.x; out[7] = in.y; out[8] = in.z;
    }
    {
        RNG rng(seed);
        Phong ph(rgb(1.0f), 20.0f);
        float3 in;
        float pdf;
        ph.sample(float3(0.3f, 0.1f, 0.9f), in, rng, pdf);   // sample_power_cos_hemisphere (brdfs.h:69)
        out[9] = in.x; out[10] = in.y; out[11] = in.z;
    }
    {
        RNG rng(seed);
        float2 d = sample_concentric_disc(rng.random_float(), rng.random_float());
        out[12] = d.x; out[13] = d.y;
    }
}

// The reference-layout arrays the reference's adapters wrote (GPU two-wide layout).
int ref_scene_gpu_layout(void* h, int* root, const void** nodes, const void** insts, const void** tris,
                         int64_t* sizes) {
    RefScene* rs = static_cast<RefScene*>(h);
    const auto& td = rs->scene.traversal_data_gpu();
    *root = td.root;
    *nodes = td.nodes.data();
    *insts = td.instances.data();
    *tris = td.tris.data();
    sizes[0] = td.nodes.size();
    sizes[1] = td.instances.size();
    sizes[2] = td.tris.size();
    return 0;
}

// The four-wide CPU layout (scenes created after ref_set_next_scene_options(1, ...)).
int ref_scene_cpu_layout(void* h, int* root, const void** nodes, const void** insts, const void** tris,
                         int64_t* sizes) {
    RefScene* rs = static_cast<RefScene*>(h);
    if (!rs->scene.has_cpu_buffers()) return -1;
    const auto& td = rs->scene.traversal_data_cpu();
    *root = td.root;
    *nodes = td.nodes.data();
    *insts = td.instances.data();
    *tris = td.tris.data();
    sizes[0] = td.nodes.size();
    sizes[1] = td.instances.size();
    sizes[2] = td.tris.size();
    return 0;
}

void ref_set_next_scene_options(int cpu_buffers, int n_files, const char* const* files) {
    g_next_cpu_buffers = cpu_buffers != 0;
    g_next_accel_files.clear();
    for (int i = 0; i < n_files; ++i) g_next_accel_files.emplace_back(files[i] ? files[i] : "");
}

// The reference's load_accel_gpu / store_accel_gpu (load_bvh.cpp) on arrays: `pre` nodes and
// Vec4s stand for other meshes already in the arrays.
int ref_load_accel(int cpu, const char* path, int tri_id_offset, const void* pre_nodes, int n_pre_nodes,
                   const float* pre_tris, int n_pre_tris, void* nodes_out, int nodes_cap, int* n_nodes,
                   float* tris_out, int tris_cap, int* n_tris) {
    auto run = [&](auto* node_tag, auto load) -> int {
        using Node = std::remove_pointer_t<decltype(node_tag)>;
        std::vector<Node> nodes((const Node*)pre_nodes, (const Node*)pre_nodes + n_pre_nodes);
        std::vector<Vec4> tris((const Vec4*)pre_tris, (const Vec4*)pre_tris + n_pre_tris);
        if (!load(path, nodes, tris, tri_id_offset)) return 1;
        if ((int)nodes.size() > nodes_cap || (int)tris.size() > tris_cap) return 2;
        std::memcpy(nodes_out, nodes.data(), sizeof(Node) * nodes.size());
        std::memcpy(tris_out, tris.data(), sizeof(Vec4) * tris.size());
        *n_nodes = (int)nodes.size();
        *n_tris = (int)tris.size();
        return 0;
    };
    if (cpu) return run((traversal_cpu::Node*)nullptr, imba::load_accel_cpu);
    return run((traversal_gpu::Node*)nullptr, imba::load_accel_gpu);
}

int ref_store_accel(int cpu, const char* path, const void* nodes, int node_offset, int n_nodes, const float* tris,
                    int tris_offset, int n_tris, int tri_id_offset) {
    auto run = [&](auto* node_tag, auto store) -> int {
        using Node = std::remove_pointer_t<decltype(node_tag)>;
        std::vector<Node> nv((const Node*)nodes, (const Node*)nodes + n_nodes);
        std::vector<Vec4> tv((const Vec4*)tris, (const Vec4*)tris + n_tris);
        return store(path, nv, node_offset, tv, tris_offset, tri_id_offset) ? 0 : 1;
    };
    if (cpu) return run((traversal_cpu::Node*)nullptr, imba::store_accel_cpu);
    return run((traversal_gpu::Node*)nullptr, imba::store_accel_gpu);
}

void ref_scene_bsphere(void* h, float* out4) {
    const BSphere& s = static_cast<RefScene*>(h)->scene.bounding_sphere();
    out4[0] = s.center.x; out4[1] = s.center.y; out4[2] = s.center.z; out4[3] = s.radius;
}

// One frame of the reference path tracer (pt.cpp) with the TileScheduler: one tile covering
// the image (tile-local sample indices are then global, ray_gen.h:51-56), `threads` tile
// threads, `spp` samples per pixel, seed_base for the frame's queue fill. image_out: w*h*3.
int ref_render_pt(void* h, int w, int ht, const float* pos, const float* dir, const float* up, float fov, int spp,
                  int max_path_len, uint64_t seed_base, float* image_out) {
    RefScene* rs = static_cast<RefScene*>(h);
    use_scene_masks(rs->scene);
    PerspectiveCamera cam((float)w, (float)ht, fov);
    cam.move(f3(pos), f3(dir), f3(up));
    const int tile = w > ht ? w : ht;
    DefaultTileGen<PTState> gen(w, ht, spp, tile);
    TileScheduler<PTState, ShadowState, false> sched(gen, rs->scene, 1, 1, tile * tile * spp, true);
    PathTracer pt(rs->scene, cam, sched, max_path_len);
    AtomicImage img(w, ht);
    img.clear();
    imbart_ref_set_seed(seed_base, 0);
    pt.render(img);
    for (int i = 0; i < w * ht; ++i) {
        image_out[3 * i + 0] = img.pixels()[i][0];
        image_out[3 * i + 1] = img.pixels()[i][1];
        image_out[3 * i + 2] = img.pixels()[i][2];
    }
    return 0;
}

extern "C" imba::Integrator* imbart_make_pt_rr(imba::Scene& scene, imba::PerspectiveCamera& cam,
                                              imba::RayScheduler<imba::PTState, imba::ShadowState>& sched,
                                              int max_path_len, int rr_start);

// The reference path tracer with its Russian roulette deferred to bounce rr_start
// (ref_pt_rr.cpp), otherwise as ref_render_pt.
extern "C" int ref_render_pt_rr(void* h, int w, int ht, const float* pos, const float* dir, const float* up,
                                float fov, int spp, int max_path_len, int rr_start, uint64_t seed_base,
                                float* image_out) {
    RefScene* rs = static_cast<RefScene*>(h);
    use_scene_masks(rs->scene);
    PerspectiveCamera cam((float)w, (float)ht, fov);
    cam.move(f3(pos), f3(dir), f3(up));
    const int tile = w > ht ? w : ht;
    DefaultTileGen<PTState> gen(w, ht, spp, tile);
    TileScheduler<PTState, ShadowState, false> sched(gen, rs->scene, 1, 1, tile * tile * spp, true);
    std::unique_ptr<Integrator> pt(imbart_make_pt_rr(rs->scene, cam, sched, max_path_len, rr_start));
    AtomicImage img(w, ht);
    img.clear();
    imbart_ref_set_seed(seed_base, 0);
    pt->render(img);
    for (int i = 0; i < w * ht; ++i)
        for (int k = 0; k < 3; ++k) image_out[3 * i + k] = img.pixels()[i][k];
    return 0;
}

// The reference path tracer as its CPU baseline runs it: `threads` TileScheduler threads on
// tiles of `tile` pixels, traversal by the oracle on the calling thread of each tile. Ray
// counts are the reference TileScheduler's own statistics (tile_scheduler.h:117-127), which
// it prints when destroyed (:59-60); the harness reads that line from stdout.
int ref_render_pt_threads(void* h, int w, int ht, const float* pos, const float* dir, const float* up, float fov,
                          int spp, int max_path_len, uint64_t seed_base, int tile, int threads, float* image_out,
                          long long* counts) {
    RefScene* rs = static_cast<RefScene*>(h);
    use_scene_masks(rs->scene);
    PerspectiveCamera cam((float)w, (float)ht, fov);
    cam.move(f3(pos), f3(dir), f3(up));
    DefaultTileGen<PTState> gen(w, ht, spp, tile);
    auto* sched = new TileScheduler<PTState, ShadowState, true>(gen, rs->scene, 1, threads, tile * tile * spp, true);
    AtomicImage img(w, ht);
    img.clear();
    {
        PathTracer pt(rs->scene, cam, *sched, max_path_len);
        imbart_ref_set_seed(seed_base, 0);
        pt.render(img);
    }
    // Capture the statistics line printed by the scheduler's destructor.
    fflush(stdout);
    std::cout.flush();
    char path[] = "/tmp/imbart_ref_statsXXXXXX";
    const int fd = mkstemp(path);
    const int saved = dup(1);
    dup2(fd, 1);
    delete sched;
    std::cout.flush();
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
    lseek(fd, 0, SEEK_SET);
    char buf[256] = {0};
    const ssize_t got = read(fd, buf, sizeof(buf) - 1);
    close(fd);
    unlink(path);
    long long prim = -1, shadow = -1;
    if (got > 0) sscanf(buf, "%lld primary ray(s), %lld shadow ray(s)", &prim, &shadow);
    counts[0] = prim;
    counts[1] = shadow;
    if (image_out)
        for (int i = 0; i < w * ht; ++i)
            for (int k = 0; k < 3; ++k) image_out[3 * i + k] = img.pixels()[i][k];
    return prim >= 0 ? 0 : -1;
}

}  // extern "C"
