/*
 * Oracle: CPU restatement of closest-hit / any-hit traversal of the reference's two-level
 * instanced BVH. TEST INFRASTRUCTURE ONLY — it checks libimbart and times the CPU baseline;
 * the product never links or calls it.
 *
 * The reference's traversal lives in the external AnyDSL/traversal project, which is not
 * part of the reference tree (src/imbatracer/core/traversal_interface.h:4-10, CMakeLists.txt:34),
 * so this file restates it from the boundary the reference does contain:
 *   - entry points and buffers: src/imbatracer/render/scheduling/ray_queue.h:247-343
 *   - ray convention (tmin in org.w, tmax in dir.w): render/ray_gen/camera.h:57-65, pt.cpp:37-41
 *   - hit convention (tri_id -1 = miss, u weights v1): render/integrators/integrator.h:71-94,
 *     core/common.h:52-54, ray_queue.h:168
 *   - two-wide node and triangle-run layout: core/gpu_adapter.cpp:14-31, 62-143
 *   - instance nodes and the world-to-object transform: core/cpu_adapter.cpp:346-365,
 *     core/float3x4.h:36-40 (float3x4 * float4 evaluated left to right)
 *   - opacity masks: core/mask.h:9-40, render/scene.cpp:89-93 (material in indices[4*tri+3])
 * The triangle test is the published watertight test (Woop, Benthin, Wald, JCGT 2013) with
 * its double-precision edge fallback; ties in t resolve to the smallest (inst_id, tri_id).
 * Parity against the original AnyDSL kernels is UNPINNED (their source is absent); the GPU
 * path is checked against this restatement, which is itself checked by brute force.
 *
 * Build with -ffp-contract=off: every float operation is rounded separately, matching the
 * reference's x86-64 SSE code (no FMA in the reference build flags) and the GPU kernel's
 * explicit round-to-nearest intrinsics.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_types.h"

#define SENTINEL ((int)0x80000000)
#define DUMMY_RIGHT 0x76543210

static int fbits(float f) { union { float f; int i; } u; u.f = f; return u.i; }

typedef struct {
    float o[3], d[3];
    int kx, ky, kz;
    float Sx, Sy, Sz;
} space_t;

static int max_dim3(float x, float y, float z) { return (x > y) ? ((x > z) ? 0 : 2) : ((y > z) ? 1 : 2); }

/* Reciprocal with components below 1e-20 in magnitude replaced by +-1e-20 (keeps slab tests
 * finite, also when the kernel scales slab terms by 32768 + q). */
static float safe_rcp(float d) {
    const float tiny = 1e-20f;
    const float dd = fabsf(d) < tiny ? copysignf(tiny, d) : d;
    return 1.0f / dd;
}

/* Shear constants of the watertight test: Sz = 1/d[kz] (rounded once), Sx = d[kx] * Sz,
 * Sy = d[ky] * Sz. The paper writes the divisions d[kx]/d[kz]; any fixed definition keeps
 * the test watertight, and this one is shared with the GPU kernel. */
static void setup_shear(space_t* s) {
    const int kz = max_dim3(fabsf(s->d[0]), fabsf(s->d[1]), fabsf(s->d[2]));
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    if (s->d[kz] < 0.0f) { const int t = kx; kx = ky; ky = t; }
    s->kx = kx; s->ky = ky; s->kz = kz;
    s->Sz = safe_rcp(s->d[kz]);
    s->Sx = s->d[kx] * s->Sz;
    s->Sy = s->d[ky] * s->Sz;
}

/* Watertight test; identical operation order to the GPU kernel (trace_kernel.cuh). */
static int tri_test(const space_t* r, const float* v0, const float* v1, const float* v2,
                    float* t_out, float* u_out, float* v_out) {
    float A[3], B[3], C[3];
    for (int a = 0; a < 3; ++a) { A[a] = v0[a] - r->o[a]; B[a] = v1[a] - r->o[a]; C[a] = v2[a] - r->o[a]; }
    const float Ax = A[r->kx] - r->Sx * A[r->kz];
    const float Ay = A[r->ky] - r->Sy * A[r->kz];
    const float Bx = B[r->kx] - r->Sx * B[r->kz];
    const float By = B[r->ky] - r->Sy * B[r->kz];
    const float Cx = C[r->kx] - r->Sx * C[r->kz];
    const float Cy = C[r->ky] - r->Sy * C[r->kz];
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return 0;
    const float det = (U + V) + W;
    if (det == 0.0f) return 0;
    const float Az = r->Sz * A[r->kz];
    const float Bz = r->Sz * B[r->kz];
    const float Cz = r->Sz * C[r->kz];
    const float T = (U * Az + V * Bz) + W * Cz;
    const float rcp = 1.0f / det;
    *t_out = T * rcp;
    *u_out = V * rcp;
    *v_out = W * rcp;
    return 1;
}

static float xform_row(const float* m, float x, float y, float z, float w) {
    return ((m[0] * x + m[1] * y) + m[2] * z) + m[3] * w;
}

typedef struct {
    const int* indices;
    const o_vec2* texcoords;
    const o_mask* masks;
    const uint8_t* mask_buffer;
    int n_masks;
} mask_ctx;

static int mask_opaque(const mask_ctx* mc, int tri, float u, float v) {
    if (!mc->indices) return 1;
    const int m = mc->indices[4 * tri + 3];
    if (m < 0 || m >= mc->n_masks) return 1;
    const o_mask d = mc->masks[m];
    int x = 0, y = 0;
    if (d.width * d.height > 1) {
        const o_vec2 t0 = mc->texcoords[mc->indices[4 * tri + 0]];
        const o_vec2 t1 = mc->texcoords[mc->indices[4 * tri + 1]];
        const o_vec2 t2 = mc->texcoords[mc->indices[4 * tri + 2]];
        const float w0 = (1.0f - u) - v;
        const float tu = (t0.x * w0 + t1.x * u) + t2.x * v;
        const float tv = (t0.y * w0 + t1.y * u) + t2.y * v;
        x = (int)floorf(tu * (float)d.width) % d.width; if (x < 0) x += d.width;
        y = (int)floorf(tv * (float)d.height) % d.height; if (y < 0) y += d.height;
    }
    return mc->mask_buffer[d.offset + y * d.width + x] != 0;
}

typedef struct {
    float t, u, v;
    int tri, inst;
} best_t;

static int closer(const best_t* b, float t, int inst, int tri) {
    if (t < b->t) return 1;
    if (t == b->t) {
        if (b->tri < 0) return 1;
        if (inst < b->inst) return 1;
        if (inst == b->inst && tri < b->tri) return 1;
    }
    return 0;
}

/* Conservative slab test in double precision. The float watertight test may accept a hit a
 * few ulps of |vertex - origin| outside the exact triangle, so the box is padded by
 * 2^-18 of the magnitudes of its coordinates and of the ray origin (four times the padding
 * the GPU kernel applies): the oracle never culls a hit the triangle test would accept. */
static int box_hit(const float* o, const float* d, const o_bbox* bb, double tmin, double tmax) {
    const float lo[3] = {bb->lo_x, bb->lo_y, bb->lo_z};
    const float hi[3] = {bb->hi_x, bb->hi_y, bb->hi_z};
    double mag = 0.0;
    for (int a = 0; a < 3; ++a) {
        mag = fmax(mag, fabs((double)lo[a]));
        mag = fmax(mag, fabs((double)hi[a]));
        mag = fmax(mag, fabs((double)o[a]));
    }
    const double pad = mag * 3.814697265625e-06;
    double tn = tmin, tf = tmax;
    for (int a = 0; a < 3; ++a) {
        const double l = (double)lo[a] - pad, h = (double)hi[a] + pad;
        if (d[a] == 0.0f) {
            if (o[a] < l || o[a] > h) return 0;
            continue;
        }
        double t0 = (l - (double)o[a]) / (double)d[a];
        double t1 = (h - (double)o[a]) / (double)d[a];
        if (t0 > t1) { const double t = t0; t0 = t1; t1 = t; }
        if (t0 > tn) tn = t0;
        if (t1 < tf) tf = t1;
    }
    const double slack = 1e-9 * (fabs(tn) + fabs(tf)) + 1e-30;
    return tn <= tf + slack;
}

typedef struct {
    const o_node2* nodes;
    const o_inst* insts;
    const o_vec4* tris;
    mask_ctx mc;
    int any;
} scene2;

/* Tests a run of triangles (gpu_adapter.cpp:129-141); returns 1 to stop (any-hit found). */
static int test_run(const scene2* s, const space_t* r, int at, int inst, float tmin, best_t* b) {
    for (;;) {
        const o_vec4* t = s->tris + at;
        const float v0[3] = {t[0].x, t[0].y, t[0].z};
        const float v1[3] = {t[1].x, t[1].y, t[1].z};
        const float v2[3] = {t[2].x, t[2].y, t[2].z};
        const int id = fbits(t[1].w);
        float tt, uu, vv;
        if (tri_test(r, v0, v1, v2, &tt, &uu, &vv) && tt >= tmin && closer(b, tt, inst, id) &&
            mask_opaque(&s->mc, id, uu, vv)) {
            b->t = tt; b->u = uu; b->v = vv; b->tri = id; b->inst = inst;
            if (s->any) return 1;
        }
        if (fbits(t[2].w) == SENTINEL) return 0;
        at += 3;
    }
}

static int traverse_bottom(const scene2* s, const space_t* r, int root, int inst, float tmin, best_t* b) {
    int stack[256];
    int sp = 0;
    stack[sp++] = root;
    while (sp > 0) {
        const int n = stack[--sp];
        const o_node2* nd = s->nodes + n;
        const int kids[2] = {nd->left, nd->right};
        const o_bbox* bbs[2] = {&nd->left_bb, &nd->right_bb};
        for (int k = 0; k < 2; ++k) {
            if (k == 1 && kids[1] == DUMMY_RIGHT) continue;
            if (!box_hit(r->o, r->d, bbs[k], tmin, (double)b->t * (1.0 + 1e-6))) continue;
            if (kids[k] < 0) {
                if (test_run(s, r, ~kids[k], inst, tmin, b)) return 1;
            } else {
                if (sp >= 256) abort();
                stack[sp++] = kids[k];
            }
        }
    }
    return 0;
}

static void trace_one2(const scene2* s, int root, const o_ray* ray, o_hit* hit, float* v_out) {
    best_t b;
    b.t = ray->dir.w; b.u = 0.0f; b.v = 0.0f; b.tri = -1; b.inst = -1;
    const float tmin = ray->org.w;
    const int valid = (tmin <= b.t) && (ray->dir.x != 0.0f || ray->dir.y != 0.0f || ray->dir.z != 0.0f);
    if (valid) {
        space_t w;
        w.o[0] = ray->org.x; w.o[1] = ray->org.y; w.o[2] = ray->org.z;
        w.d[0] = ray->dir.x; w.d[1] = ray->dir.y; w.d[2] = ray->dir.z;
        int stack[256];
        int sp = 0;
        stack[sp++] = root;
        int stop = 0;
        while (sp > 0 && !stop) {
            const int n = stack[--sp];
            const o_node2* nd = s->nodes + n;
            const int kids[2] = {nd->left, nd->right};
            const o_bbox* bbs[2] = {&nd->left_bb, &nd->right_bb};
            for (int k = 0; k < 2 && !stop; ++k) {
                if (k == 1 && kids[1] == DUMMY_RIGHT) continue;
                if (!box_hit(w.o, w.d, bbs[k], tmin, (double)b.t * (1.0 + 1e-6))) continue;
                if (kids[k] >= 0) { if (sp >= 256) abort(); stack[sp++] = kids[k]; continue; }
                /* Instance run closed by pad[0] == -1. */
                for (int i = ~kids[k];; ++i) {
                    const o_inst* in = s->insts + i;
                    space_t r;
                    for (int a = 0; a < 3; ++a) {
                        r.o[a] = xform_row(in->transf + 4 * a, w.o[0], w.o[1], w.o[2], 1.0f);
                        r.d[a] = xform_row(in->transf + 4 * a, w.d[0], w.d[1], w.d[2], 0.0f);
                    }
                    setup_shear(&r);
                    if (traverse_bottom(s, &r, in->next, in->id, tmin, &b)) { stop = 1; break; }
                    if (in->pad[0] == -1) break;
                }
            }
        }
    }
    hit->tri_id = b.tri;
    hit->inst_id = b.tri >= 0 ? b.inst : -1;
    hit->tmax = b.t;
    hit->u = b.tri >= 0 ? b.u : 0.0f;
    if (v_out) *v_out = b.tri >= 0 ? b.v : 0.0f;
}

/* Traces `count` rays over the two-wide layout. Masks may be NULL (all opaque). */
void oracle_trace_node2(int root, const o_node2* nodes, const o_inst* insts, const o_vec4* tris,
                        const int* indices, const o_vec2* texcoords, const o_mask* masks, int n_masks,
                        const uint8_t* mask_buffer, const o_ray* rays, o_hit* hits, float* v_out,
                        int count, int any, int threads) {
    scene2 s;
    s.nodes = nodes; s.insts = insts; s.tris = tris; s.any = any;
    s.mc.indices = masks ? indices : NULL; s.mc.texcoords = texcoords; s.mc.masks = masks;
    s.mc.mask_buffer = mask_buffer; s.mc.n_masks = n_masks;
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads)
    for (int i = 0; i < count; ++i) trace_one2(&s, root, rays + i, hits + i, v_out ? v_out + i : NULL);
}

/* Brute force over an explicit list of instances: every triangle of every instance's mesh
 * (given as a flat triangle list per mesh) is tested. Used to check the BVH walks. */
void oracle_trace_brute(const float* mesh_tris, const int* mesh_tri_ids, const int* mesh_first,
                        const int* mesh_count, const float* inv_mats, const int* inst_mesh, int n_inst,
                        const o_ray* rays, o_hit* hits, float* v_out, int count, int any, int threads) {
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int i = 0; i < count; ++i) {
        const o_ray* ray = rays + i;
        best_t b;
        b.t = ray->dir.w; b.u = 0.0f; b.v = 0.0f; b.tri = -1; b.inst = -1;
        const float tmin = ray->org.w;
        const int valid = (tmin <= b.t) && (ray->dir.x != 0.0f || ray->dir.y != 0.0f || ray->dir.z != 0.0f);
        for (int k = 0; valid && k < n_inst; ++k) {
            space_t r;
            const float* m = inv_mats + 12 * k;
            const float wo[3] = {ray->org.x, ray->org.y, ray->org.z};
            const float wd[3] = {ray->dir.x, ray->dir.y, ray->dir.z};
            for (int a = 0; a < 3; ++a) {
                r.o[a] = xform_row(m + 4 * a, wo[0], wo[1], wo[2], 1.0f);
                r.d[a] = xform_row(m + 4 * a, wd[0], wd[1], wd[2], 0.0f);
            }
            setup_shear(&r);
            const int mesh = inst_mesh[k];
            int stop = 0;
            for (int t = mesh_first[mesh]; t < mesh_first[mesh] + mesh_count[mesh]; ++t) {
                const float* v = mesh_tris + 9 * t;
                float tt, uu, vv;
                if (tri_test(&r, v, v + 3, v + 6, &tt, &uu, &vv) && tt >= tmin &&
                    closer(&b, tt, k, mesh_tri_ids[t])) {
                    b.t = tt; b.u = uu; b.v = vv; b.tri = mesh_tri_ids[t]; b.inst = k;
                    if (any) { stop = 1; break; }
                }
            }
            if (stop) break;
        }
        hits[i].tri_id = b.tri;
        hits[i].inst_id = b.tri >= 0 ? b.inst : -1;
        hits[i].tmax = b.t;
        hits[i].u = b.tri >= 0 ? b.u : 0.0f;
        if (v_out) v_out[i] = b.tri >= 0 ? b.v : 0.0f;
    }
}

/* ------------------------------------------------------------------------------------- */
/* Byte accounting: a faithful restatement of the GPU kernel's walk over the 8-wide layout */
/* (same slab arithmetic, slot order and stack discipline), counting the bytes it fetches: */
/* 80 per node, 48 per tested triangle, 64 per entered instance, plus 32 (ray) + 16 (hit). */
/* It also returns the hit, which must equal the two-wide oracle's.                         */
/* ------------------------------------------------------------------------------------- */

#define W_SLACK 1.00000095367431640625f

typedef struct {
    float o[3], d[3], i[3];
    float pad;
    unsigned oct;
    space_t sh;
} wspace_t;

static void wsetup(wspace_t* r) {
    r->pad = fmaxf(fmaxf(fabsf(r->o[0]), fabsf(r->o[1])), fabsf(r->o[2])) * 9.5367431640625e-07f;
    for (int a = 0; a < 3; ++a) { r->i[a] = safe_rcp(r->d[a]); r->sh.o[a] = r->o[a]; r->sh.d[a] = r->d[a]; }
    r->oct = (r->d[0] < 0.0f ? 1u : 0u) | (r->d[1] < 0.0f ? 2u : 0u) | (r->d[2] < 0.0f ? 4u : 0u);
    setup_shear(&r->sh);
}

static unsigned popc8(unsigned x) { return (unsigned)__builtin_popcount(x); }
static unsigned ffs0(unsigned x) { return (unsigned)__builtin_ctz(x); }

static void wnode_hit(const o_wnode* n, const wspace_t* r, float tmin, float tlimit,
                      unsigned* hits8, unsigned* prim_mask) {
    const float s[3] = {ldexpf(1.0f, (int)n->ex - 127), ldexpf(1.0f, (int)n->ey - 127), ldexpf(1.0f, (int)n->ez - 127)};
    const float p[3] = {n->px, n->py, n->pz};
    const uint8_t* lo[3] = {n->qlo_x, n->qlo_y, n->qlo_z};
    const uint8_t* hi[3] = {n->qhi_x, n->qhi_y, n->qhi_z};
    float ax[3], bn[3], bf[3];
    for (int a = 0; a < 3; ++a) {
        ax[a] = s[a] * r->i[a];
        const float bl = (p[a] - r->pad - r->o[a]) * r->i[a];
        const float bh = (p[a] + r->pad - r->o[a]) * r->i[a];
        bn[a] = r->i[a] < 0.0f ? bh : bl;
        bf[a] = r->i[a] < 0.0f ? bl : bh;
    }
    *hits8 = 0; *prim_mask = 0;
    for (int sl = 0; sl < 8; ++sl) {
        float tn[3], tf[3];
        for (int a = 0; a < 3; ++a) {
            const uint8_t qn = r->i[a] < 0.0f ? hi[a][sl] : lo[a][sl];
            const uint8_t qf = r->i[a] < 0.0f ? lo[a][sl] : hi[a][sl];
            tn[a] = fmaf(32768.0f + (float)qn, ax[a], bn[a]);
            tf[a] = fmaf(32768.0f + (float)qf, ax[a], bf[a]);
        }
        const float tnear = fmaxf(fmaxf(tn[0], tn[1]), fmaxf(tn[2], tmin));
        const float tfar = fminf(fminf(tf[0], tf[1]), tf[2]) * W_SLACK;
        if (tnear <= fminf(tfar, tlimit)) {
            if ((n->imask >> sl) & 1u) *hits8 |= 1u << (sl ^ r->oct);
            else {
                const unsigned meta = n->meta[sl];
                *prim_mask |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);
            }
        }
    }
}

/* Returns bytes fetched by the GPU kernel for one ray; writes the hit. */
/* A scene whose top level is a single instance with the identity transform (all 12 matrix
 * entries exactly 1 or 0): the kernel starts every ray in that instance's tree directly, with
 * the object-space ray the instance entry computes, so hits are unchanged; the top-level node
 * step and the instance entry are skipped (counts). */
static int identity_inst(const o_winst* in) {
    for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 4; ++c)
            if (in->m[4 * a + c] != (a == c ? 1.0f : 0.0f)) return 0;
    return 1;
}

static int64_t wide_one(const o_wnode* nodes, const o_wtri* tris, const o_winst* insts, int root,
                        const o_ray* ray, int any, o_hit* hit, int64_t* counts, const o_winst* direct) {
    int64_t bytes = 32 + 16;
    best_t b;
    b.t = ray->dir.w; b.u = 0.0f; b.v = 0.0f; b.tri = -1; b.inst = -1;
    const float tmin = ray->org.w;
    const int valid = (tmin <= b.t) && (ray->dir.x != 0.0f || ray->dir.y != 0.0f || ray->dir.z != 0.0f);
    if (valid) {
        wspace_t world, r;
        world.o[0] = ray->org.x; world.o[1] = ray->org.y; world.o[2] = ray->org.z;
        world.d[0] = ray->dir.x; world.d[1] = ray->dir.y; world.d[2] = ray->dir.z;
        const int start_direct = direct != 0;
        if (start_direct) {
            const float o0 = world.o[0], o1 = world.o[1], o2 = world.o[2];
            const float d0 = world.d[0], d1 = world.d[1], d2 = world.d[2];
            for (int a = 0; a < 3; ++a) {
                world.o[a] = xform_row(direct->m + 4 * a, o0, o1, o2, 1.0f);
                world.d[a] = xform_row(direct->m + 4 * a, d0, d1, d2, 0.0f);
            }
        }
        wsetup(&world);
        r = world;
        int bottom = 0, cur_inst = -1;
        float tlimit = b.t * W_SLACK;
        unsigned stack_x[64], stack_y[64];
        int sp = 0;
        unsigned g_base = (unsigned)root, g_imask = 1u, g_hits = 1u << (0u ^ r.oct);
        if (start_direct) { bottom = 1; cur_inst = direct->id; g_base = (unsigned)direct->root; }
        unsigned t_base = 0, t_mask = 0;
        int done = 0;
        while (!done) {
            if (t_mask == 0 && g_hits != 0) {
                const unsigned bitpos = ffs0(g_hits);
                g_hits &= g_hits - 1;
                const unsigned slot = bitpos ^ r.oct;
                const unsigned idx = g_base + popc8(g_imask & ((1u << slot) - 1u));
                if (g_hits != 0) { if (sp == 64) break; stack_x[sp] = g_base; stack_y[sp] = (g_hits << 8) | g_imask; sp++; }
                const o_wnode* n = nodes + idx;
                bytes += 80; counts[0]++;
                unsigned h8, pm;
                wnode_hit(n, &r, tmin, tlimit, &h8, &pm);
                g_base = n->child_base; g_imask = n->imask; g_hits = h8;
                t_base = n->prim_base; t_mask = pm;
            }
            if (t_mask != 0) {
                if (bottom) {
                    while (t_mask != 0) {
                        const unsigned i = ffs0(t_mask);
                        t_mask &= t_mask - 1;
                        const o_wtri* tr = tris + t_base + i;
                        bytes += 48; counts[1]++;
                        float tt, uu, vv;
                        if (!tri_test(&r.sh, tr->v0, tr->v1, tr->v2, &tt, &uu, &vv)) continue;
                        if (!(tt >= tmin)) continue;
                        if (!closer(&b, tt, cur_inst, tr->id)) continue;
                        b.t = tt; b.u = uu; b.v = vv; b.tri = tr->id; b.inst = cur_inst;
                        tlimit = b.t * W_SLACK;
                        if (any) { done = 1; break; }
                    }
                    if (done) break;
                } else {
                    const unsigned i = ffs0(t_mask);
                    t_mask &= t_mask - 1;
                    if (sp + 3 > 64) break;
                    if (g_hits != 0) { stack_x[sp] = g_base; stack_y[sp] = (g_hits << 8) | g_imask; sp++; }
                    if (t_mask != 0) { stack_x[sp] = t_base | (1u << 30); stack_y[sp] = t_mask; sp++; }
                    stack_x[sp] = 2u << 30; stack_y[sp] = 0; sp++;
                    t_mask = 0;
                    const o_winst* in = insts + t_base + i;
                    bytes += 64; counts[2]++;
                    for (int a = 0; a < 3; ++a) {
                        r.o[a] = xform_row(in->m + 4 * a, world.o[0], world.o[1], world.o[2], 1.0f);
                        r.d[a] = xform_row(in->m + 4 * a, world.d[0], world.d[1], world.d[2], 0.0f);
                    }
                    wsetup(&r);
                    cur_inst = in->id;
                    bottom = 1;
                    g_base = (unsigned)in->root; g_imask = 1u; g_hits = 1u << (0u ^ r.oct);
                    continue;
                }
            }
            if (g_hits == 0 && t_mask == 0) {
                for (;;) {
                    if (sp == 0) { done = 1; break; }
                    --sp;
                    const unsigned type = stack_x[sp] >> 30;
                    if (type == 2u) { r = world; bottom = 0; cur_inst = -1; continue; }
                    if (type == 1u) { t_base = stack_x[sp] & ((1u << 30) - 1u); t_mask = stack_y[sp]; break; }
                    g_base = stack_x[sp] & ((1u << 30) - 1u); g_imask = stack_y[sp] & 0xffu; g_hits = stack_y[sp] >> 8;
                    break;
                }
            }
        }
    }
    hit->tri_id = b.tri;
    hit->inst_id = b.tri >= 0 ? b.inst : -1;
    hit->tmax = b.t;
    hit->u = b.tri >= 0 ? b.u : 0.0f;
    return bytes;
}

/* Walks `count` rays over the 8-wide layout. bytes_out[i] receives ray i's fetched bytes;
 * counts_out (3 int64) accumulates visited nodes, tested triangles and entered instances. */
void oracle_wide_walk(const o_wnode* nodes, const o_wtri* tris, const o_winst* insts, int root,
                      const o_ray* rays, o_hit* hits, int64_t* bytes_out, int64_t* counts_out,
                      int count, int any, int threads, int n_insts) {
    if (threads < 1) threads = 1;
    const o_winst* direct = (n_insts == 1 && identity_inst(insts)) ? insts : 0;
    int64_t c0 = 0, c1 = 0, c2 = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads) reduction(+ : c0, c1, c2)
    for (int i = 0; i < count; ++i) {
        int64_t c[3] = {0, 0, 0};
        bytes_out[i] = wide_one(nodes, tris, insts, root, rays + i, any, hits + i, c, direct);
        c0 += c[0]; c1 += c[1]; c2 += c[2];
    }
    counts_out[0] += c0; counts_out[1] += c1; counts_out[2] += c2;
}
