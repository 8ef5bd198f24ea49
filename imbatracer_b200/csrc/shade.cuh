// Device restatement of the reference's shading math, used by the wavefront integrators.
// Compiled with -fmad=false: every + - * / rounds separately, as in the reference's x86-64
// SSE build. Where the reference passes two rng.random_float() calls as arguments of one
// call, the reference build (g++) evaluated the RIGHT argument first; the draws below are
// taken in that order (checked against the reference itself).
//
//   vectors, dot, cross, normalize           core/float3.h, core/float4.h, core/common.h
//   local_coordinates, samplers, RR          render/random.h:57-188
//   calculate_intersection                   render/integrators/integrator.h:71-123
//   BSDF frame, lobe choice, eval/pdf         render/materials/bsdf.h:125-238
//   Lambertian, SpecularReflection, Phong,   render/materials/brdfs.h:8-227
//   CookTorrance
//   SpecularTransmission                      render/materials/btdfs.h:6-65
//   Fresnel                                   render/materials/fresnel.h:7-75
//   materials (Diffuse, Mirror, Glass, Glossy) render/materials/materials.h:62-189
//   AreaEmitter, TriangleLight, EnvMap/Light  render/light.h:14-190, 361-544
#pragma once

#include <cfloat>
#include <stdint.h>

#include "rng.cuh"

namespace imbart {
namespace sh {

constexpr float kPi = 3.14159265359f;

// Single-precision sin, cos, pow, acos and atan2 as the reference's x86 build receives them
// from glibc, whose float functions return the correctly rounded value in all but rare
// cases: here the double-precision function (error far below half a float ulp) rounded once
// to float. CUDA's own float versions may differ from that by an ulp or two, which the
// shading code amplifies near grazing angles (adjoint shading-normal factors, Russian
// roulette on throughputs) until a path takes another turn. Every sampled direction goes
// through these; lobe values and pdfs, which only scale a path's weight, use CUDA's powf
// (the double pow there cost 2.4 % of the path-traced frame).
__device__ __forceinline__ float rsinf(float x) { return (float)sin((double)x); }
__device__ __forceinline__ float rcosf(float x) { return (float)cos((double)x); }
__device__ __forceinline__ float rpowf(float x, float y) { return (float)pow((double)x, (double)y); }
__device__ __forceinline__ float racosf(float x) { return (float)acos((double)x); }
__device__ __forceinline__ float ratan2f(float y, float x) { return (float)atan2((double)y, (double)x); }

struct V3 {
    float x, y, z;
    __device__ V3() {}
    __device__ V3(float a, float b, float c) : x(a), y(b), z(c) {}
    __device__ explicit V3(float a) : x(a), y(a), z(a) {}
    __device__ float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator-(V3 a) { return V3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 operator*(float a, V3 b) { return V3(a * b.x, a * b.y, a * b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float b) { return V3(a.x * b, a.y * b, a.z * b); }
__device__ __forceinline__ V3 operator/(V3 a, float b) { return V3(a.x / b, a.y / b, a.z / b); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ V3 normalize(V3 a) { return a * (1.0f / length(a)); }
__device__ __forceinline__ float sqr(float x) { return x * x; }
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }   // std::min
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }   // std::max
__device__ __forceinline__ float clampf(float a, float lo, float hi) { return (a < lo) ? lo : ((a > hi) ? hi : a); }
__device__ __forceinline__ bool is_black(V3 c) { return c.x <= 0.0f && c.y <= 0.0f && c.z <= 0.0f; }
__device__ __forceinline__ float luminance(V3 c) { return dot(c, V3(0.2126f, 0.7152f, 0.0722f)); }

// random.h:57-72
__device__ __forceinline__ void local_coordinates(V3 n, V3& tangent, V3& binormal) {
    const bool xy = fabsf(n.x) > fabsf(n.y);
    const int id0 = xy ? 0 : 1;
    const float sig = xy ? -1.0f : 1.0f;
    const float n0 = id0 == 0 ? n.x : n.y;
    const float inv_len = 1.0f / sqrtf(sqr(n0) + sqr(n.z));
    float t[3];
    t[id0] = n.z * sig * inv_len;
    t[1 - id0] = 0.0f;
    t[2] = n0 * -1.0f * sig * inv_len;
    tangent = V3(t[0], t[1], t[2]);
    binormal = cross(n, tangent);
    tangent = normalize(tangent);
    binormal = normalize(binormal);
}

__device__ __forceinline__ V3 spherical_dir(float sin_t, float cos_t, float phi) {
    return V3(sin_t * rcosf(phi), sin_t * rsinf(phi), cos_t);
}

// sample_cos_hemisphere(u1, u2) (random.h:81-84); returns pdf in *pdf.
__device__ __forceinline__ V3 sample_cos_hemisphere(float u1, float u2, float* pdf) {
    const V3 d = spherical_dir(sqrtf(1 - u2), sqrtf(u2), 2.f * kPi * u1);
    *pdf = d.z / kPi;
    return d;
}
__device__ __forceinline__ float cos_hemisphere_pdf(float c) { return fabsf(c) / kPi; }

__device__ __forceinline__ V3 sample_power_cos_hemisphere(float power, float u1, float u2, float* pdf) {
    const float phi = kPi * 2.0f * u1;
    const float cos_t = rpowf(u2, 1.0f / (power + 1.0f));
    const float sin_t = sqrtf(1.0f - sqr(cos_t));
    const V3 d = spherical_dir(sin_t, cos_t, phi);
    *pdf = (power + 1.0f) * powf(cos_t, power) * 1.0f / (2.0f * kPi);
    return d;
}
__device__ __forceinline__ float power_cos_hemisphere_pdf(float power, float c) {
    return c > 0.0f ? ((power + 1.0f) * powf(c, power) * 1.0f / (2.0f * kPi)) : 0.0f;
}

// Two draws passed as (u1, u2) in the reference: the second argument is drawn first.
__device__ __forceinline__ void draw2(Rng& rng, float& u1, float& u2) {
    u2 = rng.next_float();
    u1 = rng.next_float();
}

// sample_concentric_disc (random.h:126-155, Shirley-Chiu as in SmallVCM).
__device__ __forceinline__ void sample_concentric_disc(float u1, float u2, float& dx, float& dy) {
    float phi, r;
    const float a = 2 * u1 - 1;
    const float b = 2 * u2 - 1;
    if (a > -b) {
        if (a > b) {
            r = a;
            phi = (kPi * 0.25f) * (b / a);
        } else {
            r = b;
            phi = (kPi * 0.25f) * (2.f - (a / b));
        }
    } else {
        if (a < b) {
            r = -a;
            phi = (kPi * 0.25f) * (4.f + (b / a));
        } else {
            r = -b;
            if (b != 0) phi = (kPi * 0.25f) * (6.f - (a / b));
            else phi = 0;
        }
    }
    dx = r * rcosf(phi);
    dy = r * rsinf(phi);
}
__device__ __forceinline__ float concentric_disc_pdf() { return 1.0f / kPi; }

// ---------------------------------------------------------------------------------------
// Scene data for shading
// ---------------------------------------------------------------------------------------
enum MaterialKind { kLambert = 0, kMirror = 1, kGlass = 2, kGlossy = 3, kPhong = 4, kEmissive = 5 };

struct Material {
    int kind;
    float color[3];     // diffuse colour / mirror scale / glass transmittance
    float spec[3];      // glossy & phong specular colour / glass reflectance
    float exponent;
    float eta, kappa;
    float emission[3];  // area emitter intensity
    float area;         // area of the emissive face (object space)
    int tex;            // diffuse texture (Lambertian, glossy, Phong): index or -1
    int bump;           // bump map: texture index or -1
};

// Light kinds of light.h: triangle (TriangleLight :94-190), directional (:192-237), point
// (:239-290), spot (:292-355). The constant environment is light 0 when present.
enum LightKind { kLightTri = 0, kLightDirectional = 1, kLightPoint = 2, kLightSpot = 3 };

struct LightSrc {
    float v[3][3];      // triangle: vertices; point / spot: v[0] = position
    float normal[3], tangent[3], binormal[3];   // triangle / spot: frame of the normal; directional:
                                                // frame of the direction the light travels
    float area;         // triangle area
    float intensity[3];
    int kind;
    float cos_angle;    // spot: cos of the cone half-angle
};

struct ShadingScene {
    const float* vertices;      // 3 floats per global vertex
    const float* normals;       // 3 floats per global vertex
    const float* texcoords;     // 2 floats per global vertex
    const int4* tris;           // global vertex indices + material, per global triangle
    const float* geom_normals;  // 3 floats per global triangle
    const float* inst_inv;      // 12 floats (3x4 row-major world-to-object) per instance
    const Material* materials;
    const LightSrc* lights;     // lights in light-list order after the environment
    const float4* tex_pixels;   // texture texels (rgba), all textures back to back
    const int4* tex_info;       // per texture: first texel, width, height
    int n_textures;
    int n_materials;
    int n_lights;
    int light_count;            // environment (if any) + lights
    int has_env;
    float env_color[3];         // intensity * constant environment colour
    float bsphere[5];           // centre xyz, radius, 1/radius^2
    int env_map;                // 0: constant environment; else 1 + texture index of its image
    float env_intensity;        // scale of the environment image
};

// ---------------------------------------------------------------------------------------
// Intersection (integrator.h:71-123)
// ---------------------------------------------------------------------------------------
// TextureSampler::sample (texture_sampler.h:18-46): bilinear, wrapped, v flipped.
__device__ __forceinline__ V3 texture_sample(const ShadingScene& s, int t, float uvx, float uvy) {
    const int4 ti = s.tex_info[t];
    const int w = ti.y, h = ti.z;
    float u = clampf(uvx - (float)(int)uvx, -1.0f, 1.0f);
    float v = clampf(uvy - (float)(int)uvy, -1.0f, 1.0f);
    u += u < 0.0f ? 1.0f : 0.0f;
    v += v < 0.0f ? 1.0f : 0.0f;
    v = 1.0f - v;
    const float kx = u * (float)(w - 1);
    const float ky = v * (float)(h - 1);
    const int x0 = (int)kx;
    const int y0 = (int)ky;
    const int x1 = (x0 + 1) % w;
    const int y1 = (y0 + 1) % h;
    const float gx = kx - floorf(kx);
    const float gy = ky - floorf(ky);
    const float hx = 1.0f - gx;
    const float hy = 1.0f - gy;
    const float4* px = s.tex_pixels + ti.x;
    const float4 a = px[y0 * w + x0], b = px[y0 * w + x1], c = px[y1 * w + x0], d = px[y1 * w + x1];
    const V3 i00(a.x, a.y, a.z), i10(b.x, b.y, b.z), i01(c.x, c.y, c.z), i11(d.x, d.y, d.z);
    return hy * (hx * i00 + gx * i10) + gy * (hx * i01 + gx * i11);
}

struct Isect {
    V3 pos, out_dir, normal, geom_normal, u_tangent, v_tangent;
    float uv[2];
    int mat;
};

__device__ __forceinline__ V3 load3(const float* p, int i) { return V3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

__device__ __forceinline__ Isect calculate_intersection(const ShadingScene& s, int tri_id, int inst_id, float tmax,
                                                         float hit_u, V3 org, V3 out_dir) {
    const int4 t = s.tris[tri_id];
    const float* m = s.inst_inv + 12 * inst_id;
    Isect r;
    r.mat = t.w;
    const V3 pos = org + tmax * out_dir;
    // local_pos = inv_mat * float4(pos, 1) (float3x4.h:36-40)
    const V3 lp(m[0] * pos.x + m[1] * pos.y + m[2] * pos.z + m[3] * 1.0f,
                m[4] * pos.x + m[5] * pos.y + m[6] * pos.z + m[7] * 1.0f,
                m[8] * pos.x + m[9] * pos.y + m[10] * pos.z + m[11] * 1.0f);
    const float u = hit_u;
    const V3 v0 = load3(s.vertices, t.x);
    const V3 e1 = load3(s.vertices, t.y) - v0;
    const V3 e2 = load3(s.vertices, t.z) - v0;
    const float v = dot(lp - v0 - u * e1, e2) / dot(e2, e2);
    const float w0 = 1 - u - v;
    r.uv[0] = s.texcoords[2 * t.x] * w0 + s.texcoords[2 * t.y] * u + s.texcoords[2 * t.z] * v;
    r.uv[1] = s.texcoords[2 * t.x + 1] * w0 + s.texcoords[2 * t.y + 1] * u + s.texcoords[2 * t.z + 1] * v;
    const V3 ln = load3(s.normals, t.x) * w0 + load3(s.normals, t.y) * u + load3(s.normals, t.z) * v;
    // float3 * float3x4 (float3x4.h:43-48): the transposed product, used for normals.
    auto tmul = [&](V3 a) {
        return V3(m[0] * a.x + m[4] * a.y + m[8] * a.z, m[1] * a.x + m[5] * a.y + m[9] * a.z,
                  m[2] * a.x + m[6] * a.y + m[10] * a.z);
    };
    r.normal = normalize(tmul(ln));
    r.geom_normal = normalize(tmul(load3(s.geom_normals, tri_id)));
    r.out_dir = -normalize(out_dir);
    r.pos = pos;
    local_coordinates(r.normal, r.u_tangent, r.v_tangent);
    // Material::bump (materials.h:32-53): finite differences of the bump map's red channel.
    const int bump = s.materials[r.mat].bump;
    if (bump >= 0) {
        const float du = 0.001f, dv = 0.001f, vscale = 0.02f;
        const V3 u_displace = texture_sample(s, bump, r.uv[0] + du, r.uv[1]);
        const V3 v_displace = texture_sample(s, bump, r.uv[0], r.uv[1] + dv);
        const V3 displace = texture_sample(s, bump, r.uv[0], r.uv[1]);
        const float diff_u = vscale * (u_displace - displace).x / du;
        const float diff_v = vscale * (v_displace - displace).x / dv;
        const V3 nb = cross(r.v_tangent, r.u_tangent);
        const V3 ub = r.u_tangent + diff_u * nb;
        const V3 vb = r.v_tangent + diff_v * nb;
        r.u_tangent = normalize(ub);
        r.v_tangent = normalize(vb);
        r.normal = cross(r.u_tangent, r.v_tangent);
    }
    if (dot(r.geom_normal, r.normal) < 0.0f) r.normal = -r.normal;
    return r;
}

// ---------------------------------------------------------------------------------------
// BxDFs in shading space (normal = z)
// ---------------------------------------------------------------------------------------
enum Flags { kNone = 0, kRefl = 1, kTrans = 2, kDiffuse = 4, kGlossyF = 8, kSpecular = 16 };

__device__ __forceinline__ bool same_hemisphere(V3 a, V3 b) { return a.z * b.z > 0.0f; }

__device__ __forceinline__ float fresnel_conductor(float cosi, float eta, float kappa) {
    const float ekc = (eta * eta + kappa * kappa) * cosi * cosi;
    const float par = (ekc - (2.f * eta * cosi) + 1) / (ekc + (2.f * eta * cosi) + 1);
    const float ek = eta * eta + kappa * kappa;
    const float perp = (ek - (2.f * eta * cosi) + cosi * cosi) / (ek + (2.f * eta * cosi) + cosi * cosi);
    return (par + perp) / 2.f;
}

__device__ __forceinline__ float fresnel_dielectric_eval(float cosi, float eta_outside, float eta_inside) {
    float eta_in = eta_outside, eta_trans = eta_inside;
    if (cosi <= 0.0f) { const float t = eta_in; eta_in = eta_trans; eta_trans = t; }
    const float sin_trans = eta_in / eta_trans * sqrtf(smax(0.0f, 1.0f - sqr(cosi)));
    if (sin_trans >= 1.0f) return 1.0f;
    const float cos_trans = sqrtf(smax(0.0f, 1.0f - sqr(sin_trans)));
    const float ci = fabsf(cosi);
    const float par = (eta_trans * ci - eta_in * cos_trans) / (eta_trans * ci + eta_in * cos_trans);
    const float perp = (eta_in * ci - eta_trans * cos_trans) / (eta_in * ci + eta_trans * cos_trans);
    return (par * par + perp * perp) / 2.f;
}

// Lambertian (brdfs.h:8-21)
__device__ __forceinline__ V3 lambert_eval(V3 c, V3 o, V3 i) {
    return same_hemisphere(o, i) ? c * (1.0f / kPi) : V3(0.0f);
}
__device__ __forceinline__ float default_pdf(V3 o, V3 i) { return same_hemisphere(o, i) ? cos_hemisphere_pdf(i.z) : 0.0f; }
// BxDF::sample default (bsdf.h:54-64)
__device__ __forceinline__ V3 lambert_sample(V3 c, V3 o, V3& in, Rng& rng, float* pdf) {
    float u1, u2;
    draw2(rng, u1, u2);
    in = sample_cos_hemisphere(u1, u2, pdf);
    if (o.z < 0.0f) in.z = -in.z;
    return lambert_eval(c, o, in);
}

// Phong (brdfs.h:48-91)
__device__ __forceinline__ V3 phong_eval(const float* c, float e, V3 o, V3 i) {
    const V3 ri(-i.x, -i.y, i.z);
    float cos_r_o = smax(0.0f, dot(ri, o));
    cos_r_o = smin(cos_r_o, 1.0f);
    return same_hemisphere(o, i) ? (e + 2.0f) / (2.0f * kPi) * V3(c[0], c[1], c[2]) * powf(cos_r_o, e) : V3(0.0f);
}
__device__ __forceinline__ V3 phong_sample(const float* c, float e, V3 o, V3& in, Rng& rng, float* pdf) {
    float u1, u2;
    draw2(rng, u1, u2);
    float p;
    const V3 d = sample_power_cos_hemisphere(e, u1, u2, &p);
    const V3 ri(-o.x, -o.y, o.z);
    V3 rt, rb;
    local_coordinates(ri, rt, rb);
    in = V3(rb.x * d.x + rt.x * d.y + ri.x * d.z, rb.y * d.x + rt.y * d.y + ri.y * d.z,
            rb.z * d.x + rt.z * d.y + ri.z * d.z);
    *pdf = p;
    return same_hemisphere(o, in) ? phong_eval(c, e, o, in) : V3(0.0f);
}
__device__ __forceinline__ float phong_pdf(float e, V3 o, V3 i) { return power_cos_hemisphere_pdf(e, i.z); }

// CookTorrance with Blinn distribution (brdfs.h:147-227); Fresnel = conductor(1, exponent)
// as GlossyMaterial builds it (materials.h:179).
__device__ __forceinline__ float abs_cos(V3 d) { return fabsf(d.z); }
__device__ __forceinline__ V3 ct_eval(const float* c, float e, V3 o, V3 i) {
    if (abs_cos(o) == 0.0f || abs_cos(i) == 0.0f) return V3(0.0f);
    const V3 h = normalize(i + o);
    const float cos_half = dot(i, h);
    const float fr = fresnel_conductor(cos_half, 1.0f, e);
    if (!same_hemisphere(o, i)) return V3(0.0f);
    const float D = (e + 2.0f) / (2.0f * kPi) * powf(abs_cos(h), e);
    const float out_dot_half = dot(o, h);
    const float G = smin(1.0f, smin(2.0f * abs_cos(h) * abs_cos(o) / out_dot_half,
                                    2.0f * abs_cos(h) * abs_cos(i) / out_dot_half));
    return (V3(c[0], c[1], c[2]) * D * G * fr) / (4.0f * abs_cos(i) * abs_cos(o));
}
__device__ __forceinline__ V3 ct_sample(const float* c, float e, V3 o, V3& in, Rng& rng, float* pdf) {
    float r1, r2;
    draw2(rng, r1, r2);
    const float c_theta = rpowf(r1, 1.0f / (e + 1.0f));
    const float s_theta = sqrtf(smax(0.0f, 1.0f - sqr(c_theta)));
    const float phi = r2 * 2.0f * kPi;
    V3 h = spherical_dir(s_theta, c_theta, phi);
    if (!same_hemisphere(o, h)) h = -h;
    in = -o + 2.0f * dot(o, h) * h;
    if (dot(o, h) <= 0.0f) *pdf = 1.0f;
    else *pdf = (e + 1.0f) * powf(c_theta, e) / (2.0f * kPi * 4.0f * dot(o, h));
    return same_hemisphere(o, in) ? ct_eval(c, e, o, in) : V3(0.0f);
}
__device__ __forceinline__ float ct_pdf(float e, V3 o, V3 i) {
    if (!same_hemisphere(o, i)) return 0.0f;
    const V3 h = normalize(i + o);
    if (dot(o, h) <= 0.0f) return 0.0f;
    return (e + 1.0f) * powf(abs_cos(h), e) / (2.0f * kPi * 4.0f * dot(o, h));
}

// ---------------------------------------------------------------------------------------
// BSDF (bsdf.h:125-238) for the material kinds
// ---------------------------------------------------------------------------------------
enum { kAllFlags = kRefl | kTrans | kDiffuse | kGlossyF | kSpecular };

__device__ __forceinline__ bool is_specular_material(const Material& m) {
    return m.kind == kMirror || m.kind == kGlass;   // Material::is_specular (materials.h:92, 145)
}

struct Bsdf {
    const Material* m;
    V3 n, ut, vt, gn;
    bool adjoint = false;   // light paths: the glass BTDF drops the (eta_in / eta_trans)^2 factor
    V3 kd{0.0f};            // diffuse colour at the hit (the material's, or its texture's)
    __device__ V3 to_local(V3 d) const { return V3(dot(vt, d), dot(ut, d), dot(n, d)); }
    __device__ V3 to_world(V3 d) const {
        return V3(vt.x * d.x + ut.x * d.y + n.x * d.z, vt.y * d.x + ut.y * d.y + n.y * d.z,
                  vt.z * d.x + ut.z * d.y + n.z * d.z);
    }
    __device__ bool has_btdf() const { return m->kind == kGlass; }
    __device__ int brdf_flags() const {
        switch (m->kind) {
            case kMirror: case kGlass: return kSpecular | kRefl;
            case kGlossy: case kPhong: return kGlossyF | kRefl | kDiffuse;
            default: return kDiffuse | kRefl;
        }
    }
    __device__ V3 brdf_eval(V3 o, V3 i) const {
        switch (m->kind) {
            case kMirror: case kGlass: return V3(0.0f);
            case kGlossy: return 0.5f * (ct_eval(m->spec, m->exponent, o, i) + lambert_eval(kd, o, i));
            case kPhong: return 0.5f * (phong_eval(m->spec, m->exponent, o, i) + lambert_eval(kd, o, i));
            default: return lambert_eval(kd, o, i);
        }
    }
    __device__ float brdf_pdf(V3 o, V3 i) const {
        switch (m->kind) {
            case kMirror: case kGlass: return 0.0f;
            case kGlossy: return (ct_pdf(m->exponent, o, i) + default_pdf(o, i)) * 0.5f;
            case kPhong: return (phong_pdf(m->exponent, o, i) + default_pdf(o, i)) * 0.5f;
            default: return default_pdf(o, i);
        }
    }
    __device__ V3 eval(V3 out_dir, V3 in_dir) const {
        const V3 lo = to_local(out_dir), li = to_local(in_dir);
        if (dot(in_dir, gn) * dot(out_dir, gn) <= 0.0f) return V3(0.0f);   // BTDFs are all specular: eval 0
        return brdf_eval(lo, li);
    }
    __device__ float pdf(V3 out_dir, V3 in_dir) const {
        const V3 lo = to_local(out_dir), li = to_local(in_dir);
        if (dot(in_dir, gn) * dot(out_dir, gn) <= 0.0f) return 0.0f;
        return brdf_pdf(lo, li);
    }
    // Samples a direction among the lobes whose flags all lie in `allowed` (BSDF::sample,
    // bsdf.h:147-199); returns the BSDF value, sets in_dir, pdf and the sampled flags.
    __device__ V3 sample(V3 out_dir, V3& in_dir, Rng& rng, int& flags, float& pdf, int allowed = kAllFlags) const {
        const V3 lo = to_local(out_dir);
        const int bf = brdf_flags();
        const bool brdf_matches = (bf & allowed) == bf;
        const bool btdf_matches = has_btdf() && ((kTrans | kSpecular) & allowed) == (kTrans | kSpecular);
        float btdf_prob;
        if (brdf_matches && btdf_matches) btdf_prob = 1.0f - fresnel_dielectric_eval(lo.z, 1.0f, m->eta);  // importance()
        else if (brdf_matches) btdf_prob = 0.0f;
        else if (btdf_matches) btdf_prob = 1.0f;
        else { pdf = 0.0f; flags = kNone; return V3(0.0f); }
        const float rnd = rng.next_float();
        const bool use_btdf = rnd < btdf_prob;
        const float component_pdf = use_btdf ? btdf_prob : 1.0f - btdf_prob;
        V3 li, value;
        int f;
        if (use_btdf) {
            // SpecularTransmission<false>(eta_inside = eta, eta_outside = 1) (btdfs.h:19-48)
            f = kTrans | kSpecular;
            pdf = 1.0f;
            float eta_in = 1.0f, eta_trans = m->eta;
            const bool entering = lo.z > 0.0f;
            if (!entering) { const float t = eta_in; eta_in = eta_trans; eta_trans = t; }
            const float sin_in_sqr = smax(0.0f, 1.0f - sqr(lo.z));
            const float eta_frac = eta_in / eta_trans;
            const float sin_trans_sqr = sqr(eta_frac) * sin_in_sqr;
            if (sin_trans_sqr >= 1.0f) {
                li = V3(-lo.x, -lo.y, lo.z);
                value = V3(0.0f);
            } else {
                float cos_trans = sqrtf(smax(0.0f, 1.0f - sin_trans_sqr));
                if (entering) cos_trans = -cos_trans;
                li = V3(eta_frac * -lo.x, eta_frac * -lo.y, cos_trans);
                const float fr = fresnel_dielectric_eval(lo.z, 1.0f, m->eta);
                const float factor = adjoint ? 1.0f : sqr(eta_in / eta_trans);
                value = factor * (1.0f - fr) * V3(m->color[0], m->color[1], m->color[2]) / fabsf(li.z);
            }
        } else {
            f = brdf_flags();
            switch (m->kind) {
                case kMirror: case kGlass: {
                    // SpecularReflection (brdfs.h:23-46)
                    li = V3(-lo.x, -lo.y, lo.z);
                    pdf = 1.0f;
                    const float fr = m->kind == kMirror ? fresnel_conductor(lo.z, m->eta, m->kappa)
                                                        : fresnel_dielectric_eval(lo.z, 1.0f, m->eta);
                    const float* sc = m->kind == kMirror ? m->color : m->spec;
                    value = fr * V3(sc[0], sc[1], sc[2]) / fabsf(li.z);
                    break;
                }
                case kGlossy: case kPhong: {
                    // CombineBxDF::sample (bsdf.h:84-86): one draw picks the lobe; the sampled
                    // flags stay the union of both lobes' (bsdf.h:76, 185).
                    const bool first = rng.next_float() < 0.5f;
                    if (first) {
                        value = m->kind == kGlossy ? ct_sample(m->spec, m->exponent, lo, li, rng, &pdf)
                                                   : phong_sample(m->spec, m->exponent, lo, li, rng, &pdf);
                    } else {
                        value = lambert_sample(kd, lo, li, rng, &pdf);
                    }
                    break;
                }
                default:
                    value = lambert_sample(kd, lo, li, rng, &pdf);
                    break;
            }
        }
        if (pdf == 0.0f) { flags = kNone; return V3(0.0f); }
        flags = f;
        in_dir = to_world(li);
        pdf *= component_pdf;
        const float side = dot(in_dir, gn) * dot(out_dir, gn);
        if ((!use_btdf && side <= 0.0f) || (use_btdf && side >= 0.0f)) { flags = kNone; return V3(0.0f); }
        return value;
    }
};

// ---------------------------------------------------------------------------------------
// Lights
// ---------------------------------------------------------------------------------------
struct DirectSample {
    V3 dir;
    float distance;
    V3 radiance;
    float pdf_direct_w;
    float pdf_emit_w;
    float cos_out;
    bool delta;
};

// Light::EmitSample (light.h:65-80)
struct EmitSample {
    V3 pos, dir, radiance;
    float cos_out, pdf_emit_w, pdf_direct_a;
};

// TriangleLight::sample_direct (light.h:142-175)
__device__ __forceinline__ DirectSample tri_light_sample(const LightSrc& L, V3 from, Rng& rng) {
    DirectSample s;
    float r1, r2;
    draw2(rng, r1, r2);
    const float sr = sqrtf(r1);
    const float u = 1.0f - sr, v = r2 * sr;
    const V3 p0(L.v[0][0], L.v[0][1], L.v[0][2]), p1(L.v[1][0], L.v[1][1], L.v[1][2]), p2(L.v[2][0], L.v[2][1], L.v[2][2]);
    const V3 pos = u * p0 + v * p1 + (1.0f - u - v) * p2;
    V3 d = pos - from;
    const float distsq = dot(d, d);
    s.distance = sqrtf(distsq);
    s.dir = d * (1.0f / s.distance);
    const V3 n(L.normal[0], L.normal[1], L.normal[2]);
    const float cos_out = dot(n, -1.0f * s.dir);
    if (cos_out > 0.0f && cos_out < 1.0f) {
        s.radiance = V3(L.intensity[0], L.intensity[1], L.intensity[2]) * cos_out * (L.area / distsq);
        s.cos_out = cos_out;
        s.pdf_emit_w = cos_hemisphere_pdf(cos_out) / L.area;
        s.pdf_direct_w = 1.0f / L.area * distsq / cos_out;
    } else {
        s.radiance = V3(0.0f);
        s.cos_out = 1.0f;
        s.pdf_emit_w = 1.0f;
        s.pdf_direct_w = 1.0f;
    }
    s.delta = false;
    return s;
}

// The environment image's size (1 x 1 for a constant environment) and its texel at
// (x, y) = (int)(s * (w - 1)), (int)(t * (h - 1)) times its intensity: EnvMap's image lookup
// img_(s * (width - 1), t * (height - 1)) (light.h:413-424, 458-470; Image::operator()
// truncates the coordinates).
__device__ __forceinline__ void env_size(const ShadingScene& sc, int& w, int& h) {
    if (sc.env_map == 0) { w = 1; h = 1; return; }
    const int4 ti = sc.tex_info[sc.env_map - 1];
    w = ti.y;
    h = ti.z;
}

__device__ __forceinline__ V3 env_lookup(const ShadingScene& sc, float s, float t) {
    if (sc.env_map == 0) return V3(sc.env_color[0], sc.env_color[1], sc.env_color[2]);
    const int4 ti = sc.tex_info[sc.env_map - 1];
    const int x = (int)(s * (float)(ti.y - 1)), y = (int)(t * (float)(ti.z - 1));
    const float4 c = sc.tex_pixels[ti.x + y * ti.y + x];
    return sc.env_intensity * V3(c.x, c.y, c.z);
}

// EnvLight::sample_direct (light.h:446-485, 525-539): a uniform (u, v) on the map (the
// reference does not importance-sample the image).
__device__ __forceinline__ DirectSample env_light_sample(const ShadingScene& sc, Rng& rng) {
    DirectSample s;
    int w, h;
    env_size(sc, w, h);
    float pdf = 1.0f / float(w * h);
    const float ux = rng.next_float();
    const float uy = rng.next_float();
    pdf *= float(w * h);
    const V3 color = env_lookup(sc, ux, uy);
    const float theta = kPi * uy;
    const float sin_theta = rsinf(theta);
    const float phi = 2.0f * kPi * ux;
    s.dir = V3(sin_theta * rsinf(phi), rcosf(theta), sin_theta * rcosf(phi));
    if (sin_theta != 0.0f) pdf /= 2.0f * kPi * kPi * sin_theta;
    else pdf = 0.0f;
    s.distance = FLT_MAX;
    s.radiance = color / pdf;
    s.pdf_direct_w = pdf;
    s.pdf_emit_w = concentric_disc_pdf() * sc.bsphere[4] * pdf;
    s.cos_out = 1.0f;
    s.delta = false;
    return s;
}

// TriangleLight::sample_emit (light.h:109-140)
__device__ __forceinline__ EmitSample tri_light_emit(const LightSrc& L, Rng& rng) {
    EmitSample s;
    float r1, r2;
    draw2(rng, r1, r2);
    const float sr = sqrtf(r1);
    const float u = 1.0f - sr, v = r2 * sr;
    const V3 p0(L.v[0][0], L.v[0][1], L.v[0][2]), p1(L.v[1][0], L.v[1][1], L.v[1][2]), p2(L.v[2][0], L.v[2][1], L.v[2][2]);
    s.pos = u * p0 + v * p1 + (1.0f - u - v) * p2;
    float c1, c2, pdf;
    draw2(rng, c1, c2);
    const V3 d = sample_cos_hemisphere(c1, c2, &pdf);
    const V3 n(L.normal[0], L.normal[1], L.normal[2]), t(L.tangent[0], L.tangent[1], L.tangent[2]),
        b(L.binormal[0], L.binormal[1], L.binormal[2]);
    s.dir = d.x * b + d.y * t + d.z * n;
    if (pdf <= 0.0f) {
        s.radiance = V3(0.0f);
        s.cos_out = 0.0f;
        s.pdf_emit_w = 1.0f;
        s.pdf_direct_a = 1.0f;
        return s;
    }
    s.radiance = V3(L.intensity[0], L.intensity[1], L.intensity[2]) * L.area * kPi;
    s.cos_out = d.z;
    s.pdf_emit_w = pdf / L.area;
    s.pdf_direct_a = 1.0f / L.area;
    return s;
}

// EnvLight::sample_emit (light.h:494-523, 446-485): a direction from the map, then a point
// on the disc of the scene's bounding sphere facing it.
__device__ __forceinline__ EmitSample env_light_emit(const ShadingScene& sc, Rng& rng) {
    EmitSample s;
    int w, h;
    env_size(sc, w, h);
    float pdf = 1.0f / float(w * h);
    const float ux = rng.next_float();
    const float uy = rng.next_float();
    pdf *= float(w * h);
    const V3 color = env_lookup(sc, ux, uy);
    const float theta = kPi * uy;
    const float sin_theta = rsinf(theta);
    const float phi = 2.0f * kPi * ux;
    V3 dir(sin_theta * rsinf(phi), rcosf(theta), sin_theta * rcosf(phi));
    if (sin_theta != 0.0f) pdf /= 2.0f * kPi * kPi * sin_theta;
    else pdf = 0.0f;
    dir = dir * -1.0f;
    float d1, d2, dx, dy;
    draw2(rng, d1, d2);
    sample_concentric_disc(d1, d2, dx, dy);
    V3 tangent, binormal;
    local_coordinates(dir, tangent, binormal);
    const V3 c(sc.bsphere[0], sc.bsphere[1], sc.bsphere[2]);
    s.pos = c + sc.bsphere[3] * (-dir + binormal * dx + tangent * dy);
    s.dir = dir;
    s.pdf_direct_a = pdf;
    s.pdf_emit_w = concentric_disc_pdf() * sc.bsphere[4] * pdf;
    s.cos_out = 1.0f;
    s.radiance = color / s.pdf_emit_w;
    return s;
}

// DirectionalLight / PointLight / SpotLight::sample_direct (light.h:216-230, 265-282, 330-351):
// no random numbers are drawn.
__device__ __forceinline__ DirectSample delta_light_sample(const LightSrc& L, const ShadingScene& sc, V3 from) {
    DirectSample s;
    s.delta = true;
    s.cos_out = 1.0f;
    const V3 I(L.intensity[0], L.intensity[1], L.intensity[2]);
    if (L.kind == kLightDirectional) {
        s.dir = -V3(L.normal[0], L.normal[1], L.normal[2]);
        s.distance = FLT_MAX;
        s.radiance = I;
        s.pdf_direct_w = 1.0f;
        s.pdf_emit_w = concentric_disc_pdf() * sc.bsphere[4];
        return s;
    }
    V3 dir = V3(L.v[0][0], L.v[0][1], L.v[0][2]) - from;
    const float sqdist = dot(dir, dir);
    const float dist = sqrtf(sqdist);
    dir = dir * (1.0f / dist);
    s.dir = dir;
    s.distance = dist;
    s.pdf_direct_w = sqdist;
    if (L.kind == kLightPoint) {
        s.radiance = I / (4.0f * kPi * sqdist);
        s.pdf_emit_w = 1.0f / (4.0f * kPi);
    } else {   // spot
        const float cos_o = -dot(dir, V3(L.normal[0], L.normal[1], L.normal[2]));
        if (cos_o < L.cos_angle) {
            s.radiance = V3(0.0f);
            s.pdf_emit_w = 0.0f;
        } else {
            s.radiance = I / sqdist;
            s.pdf_emit_w = cos_o < L.cos_angle ? 0.0f : 1.0f / (2.0f * kPi * (1 - L.cos_angle));
        }
    }
    return s;
}

// DirectionalLight / PointLight / SpotLight::sample_emit (light.h:201-214, 246-263, 304-328).
__device__ __forceinline__ EmitSample delta_light_emit(const LightSrc& L, const ShadingScene& sc, Rng& rng) {
    EmitSample s;
    const V3 I(L.intensity[0], L.intensity[1], L.intensity[2]);
    const V3 n(L.normal[0], L.normal[1], L.normal[2]), t(L.tangent[0], L.tangent[1], L.tangent[2]),
        b(L.binormal[0], L.binormal[1], L.binormal[2]);
    float u1, u2;
    draw2(rng, u1, u2);
    s.pdf_direct_a = 1.0f;
    s.cos_out = 1.0f;
    if (L.kind == kLightDirectional) {
        float dx, dy;
        sample_concentric_disc(u1, u2, dx, dy);
        const V3 c(sc.bsphere[0], sc.bsphere[1], sc.bsphere[2]);
        s.pos = c + sc.bsphere[3] * (-n + b * dx + t * dy);
        s.dir = n;
        s.pdf_emit_w = concentric_disc_pdf() * sc.bsphere[4];
        s.radiance = I / s.pdf_emit_w;
    } else if (L.kind == kLightPoint) {
        // sample_uniform_sphere (random.h:120-127)
        const float a = 2.0f * kPi * u1;
        const float bb = 2.0f * sqrtf(u2 - sqr(u2));
        s.pos = V3(L.v[0][0], L.v[0][1], L.v[0][2]);
        s.radiance = I;
        s.dir = spherical_dir(bb, 1.0f - 2.0f * u2, a);
        s.pdf_emit_w = 1.0f / (4.0f * kPi);
    } else {
        // sample_uniform_cone (random.h:161-167)
        const float phi = 2.0f * kPi * u1;
        const float cos_t = 1.0f - u2 * (1.0f - L.cos_angle);
        const float sin_t = sqrtf(1.0f - cos_t * cos_t);
        const V3 d = spherical_dir(sin_t, cos_t, phi);
        const float pdf = 1.0f / (2.0f * kPi * (1 - L.cos_angle));
        s.pos = V3(L.v[0][0], L.v[0][1], L.v[0][2]);
        s.dir = d.x * b + d.y * t + d.z * n;
        s.radiance = I / pdf;
        s.pdf_emit_w = pdf;
    }
    return s;
}

// Light l of the scene's list (the environment first when present).
__device__ __forceinline__ DirectSample light_sample_direct(const ShadingScene& s, int l, V3 from, Rng& rng) {
    if (s.has_env && l == 0) return env_light_sample(s, rng);
    const LightSrc& L = s.lights[l - s.has_env];
    return L.kind == kLightTri ? tri_light_sample(L, from, rng) : delta_light_sample(L, s, from);
}

__device__ __forceinline__ EmitSample light_emit(const ShadingScene& s, int l, Rng& rng) {
    if (s.has_env && l == 0) return env_light_emit(s, rng);
    const LightSrc& L = s.lights[l - s.has_env];
    return L.kind == kLightTri ? tri_light_emit(L, rng) : delta_light_emit(L, s, rng);
}

// Light::is_delta / is_finite
__device__ __forceinline__ bool light_is_delta(const ShadingScene& s, int l) {
    return !(s.has_env && l == 0) && s.lights[l - s.has_env].kind != kLightTri;
}
__device__ __forceinline__ bool light_is_finite(const ShadingScene& s, int l) {
    return !(s.has_env && l == 0) && s.lights[l - s.has_env].kind != kLightDirectional;
}

// The BSDF of a surface point of material m: the diffuse colour comes from the material's
// texture when it has one (DiffuseMaterial / GlossyMaterial::get_bsdf, materials.h:76-84,
// 170-181); light paths use the adjoint form.
__device__ __forceinline__ Bsdf surface_bsdf(const ShadingScene& sc, const Material& m, V3 n, V3 ut, V3 vt, V3 gn,
                                             float uvx, float uvy, bool adjoint) {
    Bsdf b{&m, n, ut, vt, gn};
    b.adjoint = adjoint;
    b.kd = (m.tex >= 0 && (m.kind == kLambert || m.kind == kGlossy || m.kind == kPhong))
               ? texture_sample(sc, m.tex, uvx, uvy)
               : V3(m.color[0], m.color[1], m.color[2]);
    return b;
}

// AreaEmitter::radiance (light.h:22-43) with both pdfs.
__device__ __forceinline__ V3 area_emitter_radiance(const Material& m, V3 out_dir, V3 normal, float* pdf_direct_a,
                                                    float* pdf_emit_w) {
    const float cos_theta_o = dot(normal, out_dir);
    if (cos_theta_o <= 0.0f) {
        *pdf_direct_a = 1.0f;
        *pdf_emit_w = 1.0f;
        return V3(0.0f);
    }
    *pdf_direct_a = 1.0f / m.area;
    V3 tangent, binormal;
    local_coordinates(normal, tangent, binormal);
    const float lz = dot(normal, out_dir);
    *pdf_emit_w = 1.0f / m.area * cos_hemisphere_pdf(lz);
    return V3(m.emission[0], m.emission[1], m.emission[2]);
}

// EnvMap::radiance (light.h:413-424): pdf_direct_w = 1 / (2 pi^2 sin t).
__device__ __forceinline__ V3 env_radiance(const ShadingScene& sc, V3 out_dir, float* pdf_direct_w) {
    float phi = ratan2f(out_dir.x, out_dir.z);
    phi = (phi < 0.0f) ? (phi + 2.0f * kPi) : phi;
    const float s = phi / (2.0f * kPi);
    const float t = racosf(out_dir.y) / kPi;
    *pdf_direct_w = 1.0f / (2.0f * kPi * kPi * rsinf(t));
    return env_lookup(sc, s, t);
}

__device__ __forceinline__ V3 env_radiance_emit(const ShadingScene& sc, V3 out_dir, float* pdf_direct_w,
                                                float* pdf_emit_w) {
    const V3 r = env_radiance(sc, out_dir, pdf_direct_w);
    *pdf_emit_w = concentric_disc_pdf() * sc.bsphere[4] * *pdf_direct_w;
    return r;
}

// Russian roulette (random.h:183-188)
__device__ __forceinline__ bool russian_roulette(V3 thr, float rnd, float& pdf) {
    const float kill_prob = luminance(thr) * 2.0f;
    pdf = smin(1.0f, kill_prob);
    return rnd < pdf;
}

}  // namespace sh
}  // namespace imbart
