// Camera set-up on the host: the matrices of PerspectiveCamera::move
// (src/imbatracer/render/ray_gen/camera.h:27-56), computed with the same single-precision
// operations in the same order (float4x4.h: perspective :26-39, scale :41-46, translate
// :48-53, product :113-119 as row-by-column dot products summed left to right, and the
// cofactor inverse :137-184 — the published gluInvertMatrix expansion). Compiled without
// floating-point contraction, so the matrices equal the reference's bit for bit.
#include <cmath>
#include <cstring>

#include "imbart_internal.h"

namespace imbart {
namespace {

constexpr float kPi = 3.14159265359f;

struct M4 { float m[4][4]; };
struct V3 { float x, y, z; };

float dot4(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3]; }
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 neg(V3 a) { return {-a.x, -a.y, -a.z}; }
float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V3 scale3(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
V3 normalize(V3 a) { return scale3(a, 1.0f / std::sqrt(dot3(a, a))); }

M4 mul(const M4& a, const M4& b) {
    M4 t, r;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) t.m[i][j] = b.m[j][i];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) r.m[i][j] = dot4(a.m[i], t.m[j]);
    return r;
}

M4 rows(const float* r0, const float* r1, const float* r2, const float* r3) {
    M4 r;
    std::memcpy(r.m[0], r0, 16); std::memcpy(r.m[1], r1, 16); std::memcpy(r.m[2], r2, 16); std::memcpy(r.m[3], r3, 16);
    return r;
}

M4 perspective(float fov, float aspect, float znear, float zfar) {
    const float f_h = 1.0f / std::tan(fov * kPi / 360.0f);
    const float f_v = aspect / std::tan(fov * kPi / 360.0f);
    const float d = 1.0f / (znear - zfar);
    M4 r;
    std::memset(&r, 0, sizeof(r));
    r.m[0][0] = f_h;
    r.m[1][1] = -f_v;
    r.m[2][2] = (znear + zfar) * d;
    r.m[2][3] = 2.0f * znear * zfar * d;
    r.m[3][2] = -1.0f;
    return r;
}

M4 scale4(float x, float y, float z, float w) {
    M4 r;
    std::memset(&r, 0, sizeof(r));
    r.m[0][0] = x; r.m[1][1] = y; r.m[2][2] = z; r.m[3][3] = w;
    return r;
}

M4 translate4(float x, float y, float z) {
    M4 r = scale4(1.0f, 1.0f, 1.0f, 1.0f);
    r.m[0][3] = x; r.m[1][3] = y; r.m[2][3] = z;
    return r;
}

// Cofactor inverse (the gluInvertMatrix expansion): each entry is the signed sum of six
// triple products, then everything is scaled by 1/det.
M4 invert(const M4& A) {
    const float (*a)[4] = A.m;
    M4 R;
    float (*r)[4] = R.m;
    r[0][0] = +a[1][1] * a[2][2] * a[3][3] - a[1][1] * a[2][3] * a[3][2] - a[2][1] * a[1][2] * a[3][3]
              + a[2][1] * a[1][3] * a[3][2] + a[3][1] * a[1][2] * a[2][3] - a[3][1] * a[1][3] * a[2][2];
    r[1][0] = -a[1][0] * a[2][2] * a[3][3] + a[1][0] * a[2][3] * a[3][2] + a[2][0] * a[1][2] * a[3][3]
              - a[2][0] * a[1][3] * a[3][2] - a[3][0] * a[1][2] * a[2][3] + a[3][0] * a[1][3] * a[2][2];
    r[2][0] = +a[1][0] * a[2][1] * a[3][3] - a[1][0] * a[2][3] * a[3][1] - a[2][0] * a[1][1] * a[3][3]
              + a[2][0] * a[1][3] * a[3][1] + a[3][0] * a[1][1] * a[2][3] - a[3][0] * a[1][3] * a[2][1];
    r[3][0] = -a[1][0] * a[2][1] * a[3][2] + a[1][0] * a[2][2] * a[3][1] + a[2][0] * a[1][1] * a[3][2]
              - a[2][0] * a[1][2] * a[3][1] - a[3][0] * a[1][1] * a[2][2] + a[3][0] * a[1][2] * a[2][1];
    const float det = a[0][0] * r[0][0] + a[0][1] * r[1][0] + a[0][2] * r[2][0] + a[0][3] * r[3][0];
    if (det == 0) {
        std::memset(&R, 0, sizeof(R));
        return R;
    }
    r[0][1] = -a[0][1] * a[2][2] * a[3][3] + a[0][1] * a[2][3] * a[3][2] + a[2][1] * a[0][2] * a[3][3]
              - a[2][1] * a[0][3] * a[3][2] - a[3][1] * a[0][2] * a[2][3] + a[3][1] * a[0][3] * a[2][2];
    r[1][1] = +a[0][0] * a[2][2] * a[3][3] - a[0][0] * a[2][3] * a[3][2] - a[2][0] * a[0][2] * a[3][3]
              + a[2][0] * a[0][3] * a[3][2] + a[3][0] * a[0][2] * a[2][3] - a[3][0] * a[0][3] * a[2][2];
    r[2][1] = -a[0][0] * a[2][1] * a[3][3] + a[0][0] * a[2][3] * a[3][1] + a[2][0] * a[0][1] * a[3][3]
              - a[2][0] * a[0][3] * a[3][1] - a[3][0] * a[0][1] * a[2][3] + a[3][0] * a[0][3] * a[2][1];
    r[3][1] = +a[0][0] * a[2][1] * a[3][2] - a[0][0] * a[2][2] * a[3][1] - a[2][0] * a[0][1] * a[3][2]
              + a[2][0] * a[0][2] * a[3][1] + a[3][0] * a[0][1] * a[2][2] - a[3][0] * a[0][2] * a[2][1];
    r[0][2] = +a[0][1] * a[1][2] * a[3][3] - a[0][1] * a[1][3] * a[3][2] - a[1][1] * a[0][2] * a[3][3]
              + a[1][1] * a[0][3] * a[3][2] + a[3][1] * a[0][2] * a[1][3] - a[3][1] * a[0][3] * a[1][2];
    r[1][2] = -a[0][0] * a[1][2] * a[3][3] + a[0][0] * a[1][3] * a[3][2] + a[1][0] * a[0][2] * a[3][3]
              - a[1][0] * a[0][3] * a[3][2] - a[3][0] * a[0][2] * a[1][3] + a[3][0] * a[0][3] * a[1][2];
    r[2][2] = +a[0][0] * a[1][1] * a[3][3] - a[0][0] * a[1][3] * a[3][1] - a[1][0] * a[0][1] * a[3][3]
              + a[1][0] * a[0][3] * a[3][1] + a[3][0] * a[0][1] * a[1][3] - a[3][0] * a[0][3] * a[1][1];
    r[3][2] = -a[0][0] * a[1][1] * a[3][2] + a[0][0] * a[1][2] * a[3][1] + a[1][0] * a[0][1] * a[3][2]
              - a[1][0] * a[0][2] * a[3][1] - a[3][0] * a[0][1] * a[1][2] + a[3][0] * a[0][2] * a[1][1];
    r[0][3] = -a[0][1] * a[1][2] * a[2][3] + a[0][1] * a[1][3] * a[2][2] + a[1][1] * a[0][2] * a[2][3]
              - a[1][1] * a[0][3] * a[2][2] - a[2][1] * a[0][2] * a[1][3] + a[2][1] * a[0][3] * a[1][2];
    r[1][3] = +a[0][0] * a[1][2] * a[2][3] - a[0][0] * a[1][3] * a[2][2] - a[1][0] * a[0][2] * a[2][3]
              + a[1][0] * a[0][3] * a[2][2] + a[2][0] * a[0][2] * a[1][3] - a[2][0] * a[0][3] * a[1][2];
    r[2][3] = -a[0][0] * a[1][1] * a[2][3] + a[0][0] * a[1][3] * a[2][1] + a[1][0] * a[0][1] * a[2][3]
              - a[1][0] * a[0][3] * a[2][1] - a[2][0] * a[0][1] * a[1][3] + a[2][0] * a[0][3] * a[1][1];
    r[3][3] = +a[0][0] * a[1][1] * a[2][2] - a[0][0] * a[1][2] * a[2][1] - a[1][0] * a[0][1] * a[2][2]
              + a[1][0] * a[0][2] * a[2][1] + a[2][0] * a[0][1] * a[1][2] - a[2][0] * a[0][2] * a[1][1];
    const float s = 1.0f / det;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) r[i][j] = r[i][j] * s;
    return R;
}

}  // namespace
}  // namespace imbart

using namespace imbart;

extern "C" int imbart_camera_setup(const float* pos, const float* dir, const float* up, float fov, float width,
                                   float height, float aspect, float* raster_to_world, float* world_to_raster,
                                   float* img_plane_dist) {
    if (!pos || !dir || !up || !raster_to_world || !(width > 0.0f) || !(height > 0.0f)) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_camera_setup: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    V3 d = normalize(V3{dir[0], dir[1], dir[2]});
    V3 u{up[0], up[1], up[2]};
    const V3 right = normalize(cross(d, u));
    u = cross(d, right);
    const V3 p{pos[0], pos[1], pos[2]};
    const V3 local_p{dot3(u, p), dot3(neg(right), p), dot3(neg(d), p)};
    const V3 nr = neg(right), nd = neg(d);
    const float r0[4] = {u.x, u.y, u.z, -local_p.x};
    const float r1[4] = {nr.x, nr.y, nr.z, -local_p.y};
    const float r2[4] = {nd.x, nd.y, nd.z, -local_p.z};
    const float r3[4] = {0.0f, 0.0f, 0.0f, 1.0f};
    const M4 world_to_cam = rows(r0, r1, r2, r3);
    const M4 persp = perspective(fov, aspect, 0.1f, 10000.0f);
    const M4 world_to_screen = mul(persp, world_to_cam);
    const M4 screen_to_world = invert(world_to_screen);
    const M4 w2r = mul(mul(scale4(height * 0.5f, width * 0.5f, 0.0f, 1.0f), translate4(1.0f, 1.0f, 0.0f)),
                       world_to_screen);
    const M4 r2w = mul(mul(screen_to_world, translate4(-1.0f, -1.0f, 0.0f)),
                       scale4(2.0f / height, 2.0f / width, 0.0f, 1.0f));
    std::memcpy(raster_to_world, r2w.m, sizeof(float) * 16);
    if (world_to_raster) std::memcpy(world_to_raster, w2r.m, sizeof(float) * 16);
    if (img_plane_dist) {
        const float tan_half = std::tan(fov * kPi / 360.0f);
        *img_plane_dist = width / (2.0f * tan_half);
    }
    return 0;
}

extern "C" int imbart_camera_make(const float* pos, const float* dir, const float* up, float fov, int width,
                                  int height, imbart_camera* out) {
    if (!out || !pos || !dir || !up || width <= 0 || height <= 0) {
        set_error(IMBART_ERR_INVALID_ARGUMENT, "imbart_camera_make: invalid argument");
        return IMBART_ERR_INVALID_ARGUMENT;
    }
    const int rc = imbart_camera_setup(pos, dir, up, fov, (float)width, (float)height, 1.0f, out->raster_to_world,
                                       out->world_to_raster, &out->img_plane_dist);
    if (rc) return rc;
    // forward_ = normalize(dir) (camera.h:29-34)
    const V3 d = normalize(V3{dir[0], dir[1], dir[2]});
    out->dir[0] = d.x; out->dir[1] = d.y; out->dir[2] = d.z;
    out->pos[0] = pos[0]; out->pos[1] = pos[1]; out->pos[2] = pos[2];
    out->width = width;
    out->height = height;
    return 0;
}
