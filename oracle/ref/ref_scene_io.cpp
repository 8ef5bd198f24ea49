// Harness around the reference's scene-file frontend (frontend/build_scene.cpp,
// loaders/load_obj.cpp, load_tga.cpp), compiled in place into oracle/_ref/libref.so.
// TEST INFRASTRUCTURE ONLY: it builds a Scene from a .scene file with the reference's own
// loaders and exports the resulting arrays (meshes, instances, materials, lights, textures,
// opacity masks) so that the product's asset loader can be compared with it. Private
// members are read by compiling the reference headers with `private` / `protected` defined
// as `public` in this translation unit only (the class layouts do not change).
//
// The harness has no libpng: PNG files do not load here (load_png returns false, the
// reference then falls back to TGA and finally to its magenta "missing texture" colour), so
// scenes compared through this harness use TGA textures.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#define private public
#define protected public
#include "imbatracer/frontend/build_scene.h"
#include "imbatracer/loaders/loaders.h"
#include "imbatracer/render/materials/materials.h"
#undef private
#undef protected

namespace imba {
bool load_png(const Path&, Image&) { return false; }
}  // namespace imba

using namespace imba;

imba::Scene* ref_scene_of(void* h);
void* ref_scene_new_empty();

namespace {

int texture_index(const Scene& scene, const TextureSampler* s) {
    if (!s) return -1;
    for (size_t i = 0; i < scene.textures().size(); ++i)
        if (scene.textures()[i].get() == s) return (int)i;
    return -2;
}

void put3(float* dst, const float3& v) { dst[0] = v.x; dst[1] = v.y; dst[2] = v.z; }
void put_rgb(float* dst, const rgb& v) { dst[0] = v.x; dst[1] = v.y; dst[2] = v.z; }

}  // namespace

extern "C" {

// Builds a scene with the reference's build_scene (build_scene.cpp:548-651); cam9 receives
// pos, dir, up. The reference's progress output goes to std::cout. NULL on failure.
void* ref_scene_load(const char* path, float* cam9) {
    void* h = ref_scene_new_empty();
    Scene* scene = ref_scene_of(h);
    float3 pos, dir, up;
    if (!build_scene(Path(path), *scene, pos, dir, up)) return nullptr;
    put3(cam9, pos); put3(cam9 + 3, dir); put3(cam9 + 6, up);
    return h;
}

// Counts: meshes, vertices (all meshes), triangles (all meshes), instances, materials,
// lights, textures, texels (all textures), masks, mask buffer bytes.
void ref_scene_counts(void* h, int64_t* out) {
    const Scene* s = ref_scene_of(h);
    int64_t nv = 0, nt = 0, texels = 0;
    for (const Mesh& m : s->meshes()) { nv += m.vertex_count(); nt += m.triangle_count(); }
    for (const auto& t : s->textures()) texels += (int64_t)t->image().width() * t->image().height();
    const auto& td = s->traversal_data_gpu();
    out[0] = s->meshes().size(); out[1] = nv; out[2] = nt; out[3] = s->instances().size();
    out[4] = s->materials().size(); out[5] = s->lights().size(); out[6] = s->textures().size(); out[7] = texels;
    out[8] = td.masks.size(); out[9] = td.mask_buffer.size();
}

// Mesh arrays, concatenated over meshes: mesh_counts (vertices, triangles per mesh),
// vertices (3), normals (3), texcoords (2), indices (4, mesh-local), geometric normals (3).
void ref_scene_meshes(void* h, int* mesh_counts, float* verts, float* normals, float* texcoords, int* indices,
                      float* geom_normals) {
    const Scene* s = ref_scene_of(h);
    for (size_t k = 0; k < s->meshes().size(); ++k) {
        const Mesh& m = s->meshes()[k];
        mesh_counts[2 * k] = m.vertex_count();
        mesh_counts[2 * k + 1] = m.triangle_count();
        auto tc = m.attribute<float2>(MeshAttributes::TEXCOORDS);
        auto nr = m.attribute<float3>(MeshAttributes::NORMALS);
        auto gn = m.attribute<float3>(MeshAttributes::GEOM_NORMALS);
        for (int v = 0; v < m.vertex_count(); ++v) {
            const float4& p = m.vertices()[v];
            verts[0] = p.x; verts[1] = p.y; verts[2] = p.z; verts += 3;
            put3(normals, nr[v]); normals += 3;
            texcoords[0] = tc[v].x; texcoords[1] = tc[v].y; texcoords += 2;
        }
        for (int t = 0; t < m.triangle_count(); ++t) {
            for (int j = 0; j < 4; ++j) indices[j] = (int)m.indices()[4 * t + j];
            indices += 4;
            put3(geom_normals, gn[t]); geom_normals += 3;
        }
    }
}

// Instances: mesh id and the object-to-world matrix (a 3x4 float3x4, row-major, written as
// 4x4 with the row 0 0 0 1).
void ref_scene_instances(void* h, int* mesh_ids, float* mats) {
    const Scene* s = ref_scene_of(h);
    for (size_t i = 0; i < s->instances().size(); ++i) {
        const Mesh::Instance& in = s->instances()[i];
        mesh_ids[i] = in.id;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) mats[16 * i + 4 * r + c] = in.mat[r][c];
        for (int c = 0; c < 4; ++c) mats[16 * i + 12 + c] = c == 3 ? 1.0f : 0.0f;
    }
}

// Materials as the product's material records: kind (0 diffuse, 1 mirror, 2 glass,
// 3 glossy; +16 when the material has an area emitter) and 16 parameters: colour[3],
// specular[3], exponent, eta, kappa, emission[3], texture, bump, emitter area, 0.
int ref_scene_materials(void* h, int* kinds, float* params) {
    const Scene* s = ref_scene_of(h);
    for (size_t i = 0; i < s->materials().size(); ++i) {
        Material* m = s->materials()[i].get();
        float* p = params + 16 * i;
        std::memset(p, 0, 16 * sizeof(float));
        int kind = -1;
        p[12] = -1.0f;
        p[13] = (float)texture_index(*s, m->bump_);
        if (auto* d = dynamic_cast<DiffuseMaterial*>(m)) {
            kind = 0;
            if (d->sampler_) p[12] = (float)texture_index(*s, d->sampler_);
            else put_rgb(p, d->color_);
        } else if (auto* r = dynamic_cast<MirrorMaterial*>(m)) {
            kind = 1;
            put_rgb(p, r->scale_);
            p[7] = r->fresnel_.eta_;
            p[8] = r->fresnel_.kappa_;
        } else if (auto* g = dynamic_cast<GlassMaterial*>(m)) {
            kind = 2;
            put_rgb(p, g->transmittance_);
            put_rgb(p + 3, g->reflectance_);
            p[7] = g->eta_;
        } else if (auto* y = dynamic_cast<GlossyMaterial*>(m)) {
            kind = 3;
            if (y->diff_sampler_) p[12] = (float)texture_index(*s, y->diff_sampler_);
            else put_rgb(p, y->diffuse_color_);
            put_rgb(p + 3, y->specular_color_);
            p[6] = y->exponent_;
        }
        if (kind < 0) return -1;
        if (const AreaEmitter* e = m->emitter()) {
            kind += 16;
            put_rgb(p + 9, e->intensity);
            p[14] = e->area;
        }
        kinds[i] = kind;
    }
    return 0;
}

// Lights in the reference's order: kind (0 triangle, 1 directional, 2 point, 3 spot,
// 4 environment) and 12
// floats as the product's light records (triangle: p0, p1, p2, intensity; directional:
// direction, 6 zero, intensity; point: position, 6 zero, intensity; spot: position, axis,
// half-angle, 2 zero, intensity).
int ref_scene_lights(void* h, int* kinds, float* params) {
    const Scene* s = ref_scene_of(h);
    for (size_t i = 0; i < s->lights().size(); ++i) {
        Light* l = s->lights()[i].get();
        float* p = params + 12 * i;
        std::memset(p, 0, 12 * sizeof(float));
        if (auto* t = dynamic_cast<TriangleLight*>(l)) {
            kinds[i] = 0;
            put3(p, t->verts_[0]); put3(p + 3, t->verts_[1]); put3(p + 6, t->verts_[2]);
            put_rgb(p + 9, t->emit_.intensity);
        } else if (auto* d = dynamic_cast<DirectionalLight*>(l)) {
            kinds[i] = 1;
            put3(p, d->dir_);
            put_rgb(p + 9, d->intensity_);
        } else if (auto* q = dynamic_cast<PointLight*>(l)) {
            kinds[i] = 2;
            put3(p, q->pos_);
            put_rgb(p + 9, q->intensity_);
        } else if (auto* sp = dynamic_cast<SpotLight*>(l)) {
            kinds[i] = 3;
            put3(p, sp->pos_);
            put3(p + 3, sp->normal_);
            p[6] = sp->angle_;
            put_rgb(p + 9, sp->intensity_);
        } else if (dynamic_cast<EnvLight*>(l)) {
            kinds[i] = 4;
        } else {
            return -1;
        }
    }
    return 0;
}

// Textures: dims (width, height per texture) and texels (rgba, row-major, concatenated).
void ref_scene_textures(void* h, int* dims, float* texels) {
    const Scene* s = ref_scene_of(h);
    for (size_t i = 0; i < s->textures().size(); ++i) {
        const Image& img = s->textures()[i]->image();
        dims[2 * i] = img.width();
        dims[2 * i + 1] = img.height();
        for (int y = 0; y < img.height(); ++y)
            for (int x = 0; x < img.width(); ++x) {
                const float4& c = img(x, y);
                texels[0] = c.x; texels[1] = c.y; texels[2] = c.z; texels[3] = c.w;
                texels += 4;
            }
    }
}

// The environment image (EnvMap, light.h:361-486): returns 0 and fills dims (width,
// height), texels (rgba rows) and the intensity when the scene has one, else -1.
int ref_scene_env(void* h, int* dims, float* texels, float* intensity) {
    const Scene* s = ref_scene_of(h);
    const EnvMap* e = s->env_map();
    if (!e) return -1;
    dims[0] = e->img_.width();
    dims[1] = e->img_.height();
    *intensity = e->intensity_;
    if (texels)
        for (int y = 0; y < e->img_.height(); ++y)
            for (int x = 0; x < e->img_.width(); ++x) {
                const float4& c = e->img_(x, y);
                texels[0] = c.x; texels[1] = c.y; texels[2] = c.z; texels[3] = c.w;
                texels += 4;
            }
    return 0;
}

// Opacity masks as uploaded for traversal: descriptors (width, height, offset) and bytes.
void ref_scene_masks(void* h, int* descs, uint8_t* buffer) {
    const Scene* s = ref_scene_of(h);
    const auto& td = s->traversal_data_gpu();
    std::memcpy(descs, td.masks.data(), sizeof(int) * 3 * td.masks.size());
    std::memcpy(buffer, td.mask_buffer.data(), td.mask_buffer.size());
}

}  // extern "C"
