// Device-side traversal of the compressed 8-wide two-level BVH (closest hit and any hit).
//
// Semantics follow the reference boundary: rays carry tmin in org.w and tmax in dir.w
// (camera.h:61-64), hits report the global triangle id, the instance id, t and the
// barycentric weight u of the triangle's second vertex (integrator.h:71-94). The triangle
// test is the watertight test of Woop, Benthin and Wald (JCGT 2013) evaluated with explicit
// round-to-nearest operations (no contraction), so that the CPU oracle computes bit-identical
// t/u/v. Equal-t hits resolve to the smallest (inst_id, tri_id), which makes the result
// independent of the traversal order and of the BVH.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "imbart_internal.h"

namespace imbart {

constexpr int kStackSize = 64;
constexpr uint32_t kTypeShift = 30;
constexpr uint32_t kIndexMask = (1u << kTypeShift) - 1u;
constexpr uint32_t kEntryNode = 0u;     // node group: x = child base, y = hits << 8 | imask
constexpr uint32_t kEntryInst = 1u;     // instance group: x = prim base, y = prim mask
constexpr uint32_t kEntryMarker = 2u;   // return from an instance to the world-space ray

// Relative slack applied to slab exits and to the current hit distance when culling
// children; together with the build-time padding of quantized boxes it makes the box test
// conservative under float rounding (cf. Ize, "Robust BVH Ray Traversal", JCGT 2013).
#define IMBART_SLACK 1.00000095367431640625f  /* 1 + 2^-20 */

struct TraceParams {
    const WideNode* __restrict__ nodes;
    const WideTri* __restrict__ tris;
    const WideInst* __restrict__ insts;
    int root;
    // alpha masks (only when masked)
    const int* __restrict__ indices;
    const float2* __restrict__ texcoords;
    const int* __restrict__ masks;          // 3 ints per descriptor
    const uint8_t* __restrict__ mask_buffer;
    int n_masks;
    // rays/hits
    const float4* __restrict__ rays;        // 2 float4 per ray
    int4* __restrict__ hits;                // 1 int4 per hit (tri, inst, t bits, u bits)
    float* __restrict__ v_out;              // optional
    int count;
    // Batches over several scenes of one node pool: ray i starts at node roots[i] instead of
    // `root` (with kDirectRootBit set: in that mesh tree, as instance 0). With count_ptr set,
    // the ray count is read from device memory at kernel start (`count` is then an upper
    // bound the launch was sized for).
    const int* __restrict__ roots;
    const int* __restrict__ count_ptr;
    int* __restrict__ error_flags;          // [0]: stack overflow count
    unsigned long long* __restrict__ stats; // statistics variant: nodes, triangles, instances
    // persistent variant
    int* __restrict__ work;                 // [0]: next ray index, [1]: finished warps (self-resetting)
    int total_warps;                        // warps in the launch
    int refill_lanes;                       // refill a warp's idle lanes once this many are idle
    int postpone_lanes;                     // postpone triangle tests while fewer lanes would test
    int tri_batch;                          // per-lane kernels: triangles a lane tests per loop trip
                                            // (0: its whole group); the cooperative ones ignore it
    // A scene whose top level is one instance with the identity transform: rays start in that
    // instance's tree (wide root direct_root, instance id direct_inst), -1 otherwise. The ray
    // is transformed by the identity rows with the instance entry's arithmetic, so it is the
    // object-space ray of the full walk bit for bit and hits are unchanged; the top-level node
    // step, the instance fetch and the second ray set-up are skipped. Never with per-ray roots.
    int direct_root;
    int direct_inst;
};

constexpr uint32_t kEntryTri = 3u;      // triangle group (postponed): x = prim base, y = prim mask

// Work counters of one ray, accumulated only by the statistics variant of the kernel.
struct RayStats {
    uint32_t nodes = 0, tris = 0, insts = 0;
};

__device__ __forceinline__ int max_dim3(float x, float y, float z) {
    return (x > y) ? ((x > z) ? 0 : 2) : ((y > z) ? 1 : 2);
}

__device__ __forceinline__ float comp3(float x, float y, float z, int k) {
    return k == 0 ? x : (k == 1 ? y : z);
}

// Per-space ray data: origin, direction, safe inverse direction, octant, shear constants,
// and the slab padding `pad` (world units of the current space). The watertight test may
// accept a hit a few ulps of |vertex - origin| outside the exact triangle; padding every
// slab by 2^-20 * max|origin| (here) and every child box by 2^-20 of the node's coordinate
// magnitude (at build time) keeps such hits inside the boxes that lead to them.
struct SpaceRay {
    float pad;
    float ox, oy, oz;
    float dx, dy, dz;
    float ix, iy, iz;
    uint32_t oct;
    int kx, ky, kz;
    float Sx, Sy, Sz;
};

__device__ __forceinline__ float safe_rcp(float d) {
    // Zero components get a huge finite inverse of the right sign so that slab tests stay
    // free of 0 * inf; the triangle test uses the true direction.
    const float tiny = 1e-20f;
    const float dd = fabsf(d) < tiny ? copysignf(tiny, d) : d;
    return __frcp_rn(dd);
}

__device__ __forceinline__ void setup_space(SpaceRay& r) {
    r.pad = fmaxf(fmaxf(fabsf(r.ox), fabsf(r.oy)), fabsf(r.oz)) * 9.5367431640625e-07f;
    r.ix = safe_rcp(r.dx); r.iy = safe_rcp(r.dy); r.iz = safe_rcp(r.dz);
    r.oct = (r.dx < 0.0f ? 1u : 0u) | (r.dy < 0.0f ? 2u : 0u) | (r.dz < 0.0f ? 4u : 0u);
    const int kz = max_dim3(fabsf(r.dx), fabsf(r.dy), fabsf(r.dz));
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    const float dkz = comp3(r.dx, r.dy, r.dz, kz);
    if (dkz < 0.0f) { const int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
    // Shear constants from the (correctly rounded) reciprocal of the dominant component:
    // Sz = 1/d[kz], Sx = d[kx] * Sz, Sy = d[ky] * Sz (the oracle uses the same definition).
    r.Sz = comp3(r.ix, r.iy, r.iz, kz);
    r.Sx = __fmul_rn(comp3(r.dx, r.dy, r.dz, kx), r.Sz);
    r.Sy = __fmul_rn(comp3(r.dx, r.dy, r.dz, ky), r.Sz);
}

// Watertight ray/triangle test. Returns true and writes t/u/v when the ray's line hits the
// triangle (edges and vertices included, both faces). u weights v1 and v weights v2.
__device__ __forceinline__ bool tri_test(const SpaceRay& r, const float4 a, const float4 b, const float4 c,
                                         float& t, float& u, float& v) {
    const float Ax0 = __fsub_rn(a.x, r.ox), Ay0 = __fsub_rn(a.y, r.oy), Az0 = __fsub_rn(a.z, r.oz);
    const float Bx0 = __fsub_rn(b.x, r.ox), By0 = __fsub_rn(b.y, r.oy), Bz0 = __fsub_rn(b.z, r.oz);
    const float Cx0 = __fsub_rn(c.x, r.ox), Cy0 = __fsub_rn(c.y, r.oy), Cz0 = __fsub_rn(c.z, r.oz);
    const float Akx = comp3(Ax0, Ay0, Az0, r.kx), Aky = comp3(Ax0, Ay0, Az0, r.ky), Akz = comp3(Ax0, Ay0, Az0, r.kz);
    const float Bkx = comp3(Bx0, By0, Bz0, r.kx), Bky = comp3(Bx0, By0, Bz0, r.ky), Bkz = comp3(Bx0, By0, Bz0, r.kz);
    const float Ckx = comp3(Cx0, Cy0, Cz0, r.kx), Cky = comp3(Cx0, Cy0, Cz0, r.ky), Ckz = comp3(Cx0, Cy0, Cz0, r.kz);
    const float Ax = __fsub_rn(Akx, __fmul_rn(r.Sx, Akz));
    const float Ay = __fsub_rn(Aky, __fmul_rn(r.Sy, Akz));
    const float Bx = __fsub_rn(Bkx, __fmul_rn(r.Sx, Bkz));
    const float By = __fsub_rn(Bky, __fmul_rn(r.Sy, Bkz));
    const float Cx = __fsub_rn(Ckx, __fmul_rn(r.Sx, Ckz));
    const float Cy = __fsub_rn(Cky, __fmul_rn(r.Sy, Ckz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        // Edge case: recompute the edge functions in double precision (Woop et al., sec. 5).
        U = __double2float_rn(__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx)));
        V = __double2float_rn(__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx)));
        W = __double2float_rn(__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax)));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    const float Az = __fmul_rn(r.Sz, Akz);
    const float Bz = __fmul_rn(r.Sz, Bkz);
    const float Cz = __fmul_rn(r.Sz, Ckz);
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
    const float rcp = __fdiv_rn(1.0f, det);
    t = __fmul_rn(T, rcp);
    u = __fmul_rn(V, rcp);
    v = __fmul_rn(W, rcp);
    return true;
}

// Transforms a world-space point/vector by the instance's 3x4 matrix, in the order of
// float3x4 * float4 (float3x4.h:36-40): ((m0*x + m1*y) + m2*z) + m3*w.
__device__ __forceinline__ float xform_row(const float4 m, float x, float y, float z, float w) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m.x, x), __fmul_rn(m.y, y)), __fmul_rn(m.z, z)), __fmul_rn(m.w, w));
}

// The object-space ray of the identity instance (TraceParams::direct_root): the instance
// entry's transform with the identity rows (for finite components it is the world ray with
// -0 turned into +0).
__device__ __forceinline__ void identity_space(SpaceRay& r, const float4 ro, const float4 rd) {
    const float4 e0 = make_float4(1.0f, 0.0f, 0.0f, 0.0f), e1 = make_float4(0.0f, 1.0f, 0.0f, 0.0f),
                 e2 = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
    r.ox = xform_row(e0, ro.x, ro.y, ro.z, 1.0f);
    r.oy = xform_row(e1, ro.x, ro.y, ro.z, 1.0f);
    r.oz = xform_row(e2, ro.x, ro.y, ro.z, 1.0f);
    r.dx = xform_row(e0, rd.x, rd.y, rd.z, 0.0f);
    r.dy = xform_row(e1, rd.x, rd.y, rd.z, 0.0f);
    r.dz = xform_row(e2, rd.x, rd.y, rd.z, 0.0f);
}

// Three-input maximum / minimum (PTX ISA 8.8, sm_100): the values of fmaxf(fmaxf(a, b), c)
// and fminf(fminf(a, b), c), NaN inputs ignored as fmaxf / fminf ignore them.
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// 32768 + (byte k of w) as an exact float, with one byte permute: the byte lands in bits
// 8..15 of the float 2^15 (0x47000000), whose mantissa step there is 1. The node's origin
// is stored 32768 quanta low, so this value feeds the slab FMA directly.
__device__ __forceinline__ float byte_plane(uint32_t w, int k) {
    return __int_as_float(__byte_perm(w, 0x47000000u, 0x7604u | ((uint32_t)k << 4)));
}

// Intersects the child boxes of a node: all 8 slots, or slots 0..3 of a 4-wide node
// (kSlots = 4, whose slots are ordered by the x/y quadrant). Returns internal-child hits in
// octant order (bit slot ^ (oct & (kSlots - 1))) and the triangle/instance hit mask relative
// to prim_base.
template <int kSlots = 8, bool kPacked = true>
__device__ __forceinline__ void intersect_node(const WideNode* __restrict__ node, const SpaceRay& r,
                                               float tmin, float tlimit,
                                               uint32_t& child_base, uint32_t& imask, uint32_t& hits8,
                                               uint32_t& prim_base, uint32_t& prim_mask) {
    const uint4* q = reinterpret_cast<const uint4*>(node);
    const uint4 q0 = __ldg(q + 0);
    const uint4 q1 = __ldg(q + 1);
    uint4 qx = __ldg(q + 2);
    uint4 qy = __ldg(q + 3);
    uint4 qz = __ldg(q + 4);
    const float sx = __uint_as_float((q0.w & 0xffu) << 23);
    const float sy = __uint_as_float(((q0.w >> 8) & 0xffu) << 23);
    const float sz = __uint_as_float(((q0.w >> 16) & 0xffu) << 23);
    imask = q0.w >> 24;
    child_base = q1.x;
    prim_base = q1.y;
    const float ax = sx * r.ix, ay = sy * r.iy, az = sz * r.iz;
    // Slab offsets of the padded low (-pad) and high (+pad) planes; the near plane is the
    // low one for positive directions.
    const float px = __uint_as_float(q0.x), py = __uint_as_float(q0.y), pz = __uint_as_float(q0.z);
    const float blx = (px - r.pad - r.ox) * r.ix, bhx = (px + r.pad - r.ox) * r.ix;
    const float bly = (py - r.pad - r.oy) * r.iy, bhy = (py + r.pad - r.oy) * r.iy;
    const float blz = (pz - r.pad - r.oz) * r.iz, bhz = (pz + r.pad - r.oz) * r.iz;
    const float bnx = r.ix < 0.0f ? bhx : blx, bfx = r.ix < 0.0f ? blx : bhx;
    const float bny = r.iy < 0.0f ? bhy : bly, bfy = r.iy < 0.0f ? bly : bhy;
    const float bnz = r.iz < 0.0f ? bhz : blz, bfz = r.iz < 0.0f ? blz : bhz;
    // Near plane uses the low bytes for positive directions, the high bytes otherwise.
    if (r.ix < 0.0f) { uint32_t t0 = qx.x, t1 = qx.y; qx.x = qx.z; qx.y = qx.w; qx.z = t0; qx.w = t1; }
    if (r.iy < 0.0f) { uint32_t t0 = qy.x, t1 = qy.y; qy.x = qy.z; qy.y = qy.w; qy.z = t0; qy.w = t1; }
    if (r.iz < 0.0f) { uint32_t t0 = qz.x, t1 = qz.y; qz.x = qz.z; qz.y = qz.w; qz.z = t0; qz.w = t1; }
    uint32_t hitbits = 0;
    // kPacked: near and far planes of an axis in one packed FMA (the same correctly rounded
    // fmaf per half). Either way the slab intervals' ends come from three-input min / max:
    // the values of fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin)) and fminf(fminf(tfx, tfy), tfz).
    // (Measured: packed is 2-4 % faster for closest hits, scalar 1-2 % for any hit.)
    const float2 a2x = make_float2(ax, ax), a2y = make_float2(ay, ay), a2z = make_float2(az, az);
    const float2 b2x = make_float2(bnx, bfx), b2y = make_float2(bny, bfy), b2z = make_float2(bnz, bfz);
#pragma unroll
    for (int s = 0; s < kSlots; ++s) {
        const uint32_t wn_x = s < 4 ? qx.x : qx.y, wf_x = s < 4 ? qx.z : qx.w;
        const uint32_t wn_y = s < 4 ? qy.x : qy.y, wf_y = s < 4 ? qy.z : qy.w;
        const uint32_t wn_z = s < 4 ? qz.x : qz.y, wf_z = s < 4 ? qz.z : qz.w;
        const int k = s & 3;
        float2 tx, ty, tz;
        if (kPacked) {
            tx = __ffma2_rn(make_float2(byte_plane(wn_x, k), byte_plane(wf_x, k)), a2x, b2x);
            ty = __ffma2_rn(make_float2(byte_plane(wn_y, k), byte_plane(wf_y, k)), a2y, b2y);
            tz = __ffma2_rn(make_float2(byte_plane(wn_z, k), byte_plane(wf_z, k)), a2z, b2z);
        } else {
            tx = make_float2(fmaf(byte_plane(wn_x, k), ax, bnx), fmaf(byte_plane(wf_x, k), ax, bfx));
            ty = make_float2(fmaf(byte_plane(wn_y, k), ay, bny), fmaf(byte_plane(wf_y, k), ay, bfy));
            tz = make_float2(fmaf(byte_plane(wn_z, k), az, bnz), fmaf(byte_plane(wf_z, k), az, bfz));
        }
        const float tn = fmax3(tx.x, ty.x, fmaxf(tz.x, tmin));
        const float tf = fmin3(tx.y, ty.y, tz.y) * IMBART_SLACK;
        hitbits |= (tn <= fminf(tf, tlimit) ? 1u : 0u) << s;
    }
    // Internal children, with bit s moved to s ^ oct (conditional bit-group swaps).
    uint32_t ib = hitbits & imask;
    if (r.oct & 1u) ib = ((ib & 0x55u) << 1) | ((ib & 0xAAu) >> 1);
    if (r.oct & 2u) ib = ((ib & 0x33u) << 2) | ((ib & 0xCCu) >> 2);
    if (kSlots == 8 && (r.oct & 4u)) ib = ((ib & 0x0Fu) << 4) | ((ib & 0xF0u) >> 4);
    hits8 = ib;
    // Leaf children: their primitive runs (count << 5 | offset in the meta byte).
    uint32_t lb = hitbits & ~imask;
    prim_mask = 0;
    while (lb != 0u) {
        const uint32_t s = __ffs(lb) - 1;
        lb &= lb - 1;
        const uint32_t meta = __byte_perm(s < 4 ? q1.z : q1.w, 0u, s & 3u) & 0xffu;
        prim_mask |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);
    }
}

// Position of the k-th (0-based) set bit of m by halving; always in [0, 31].
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, int k) {
    uint32_t pos = 0;
#pragma unroll
    for (int w = 16; w >= 1; w >>= 1) {
        const int c = __popc(m & ((1u << w) - 1u));
        if (k >= c) { k -= c; m >>= w; pos += (uint32_t)w; }
    }
    return pos;
}

// Alpha-mask lookup for a candidate hit (mask.h:22-40): transparent texels reject the hit.
__device__ __forceinline__ bool mask_opaque(const TraceParams& p, int tri, float u, float v) {
    const int m = __ldg(p.indices + 4 * tri + 3);
    if (m < 0 || m >= p.n_masks) return true;
    const int w = __ldg(p.masks + 3 * m + 0);
    const int h = __ldg(p.masks + 3 * m + 1);
    const int off = __ldg(p.masks + 3 * m + 2);
    int x = 0, y = 0;
    if (w * h > 1) {
        const float2 t0 = p.texcoords[__ldg(p.indices + 4 * tri + 0)];
        const float2 t1 = p.texcoords[__ldg(p.indices + 4 * tri + 1)];
        const float2 t2 = p.texcoords[__ldg(p.indices + 4 * tri + 2)];
        const float w0 = __fsub_rn(__fsub_rn(1.0f, u), v);
        const float tu = __fadd_rn(__fadd_rn(__fmul_rn(t0.x, w0), __fmul_rn(t1.x, u)), __fmul_rn(t2.x, v));
        const float tv = __fadd_rn(__fadd_rn(__fmul_rn(t0.y, w0), __fmul_rn(t1.y, u)), __fmul_rn(t2.y, v));
        x = (int)floorf(__fmul_rn(tu, (float)w)) % w; if (x < 0) x += w;
        y = (int)floorf(__fmul_rn(tv, (float)h)) % h; if (y < 0) y += h;
    }
    return p.mask_buffer[off + y * w + x] != 0;
}

template <bool kAnyHit, bool kMasked, bool kStats>
__device__ __forceinline__ void trace_one(const TraceParams& p, int ray_index, RayStats& st) {
    const float4 ro = __ldg(p.rays + 2 * ray_index + 0);
    const float4 rd = __ldg(p.rays + 2 * ray_index + 1);
    const float tmin = ro.w;
    const float tmax = rd.w;

    int best_tri = -1, best_inst = -1;
    float best_t = tmax, best_u = 0.0f, best_v = 0.0f;

    const bool valid = (tmin <= tmax) && (rd.x != 0.0f || rd.y != 0.0f || rd.z != 0.0f);
    if (valid) {
        const int root_word = p.roots ? __ldg(p.roots + ray_index) : p.root;
        const bool direct = p.roots ? (root_word & kDirectRootBit) != 0 : p.direct_root >= 0;
        SpaceRay world;
        world.ox = ro.x; world.oy = ro.y; world.oz = ro.z;
        world.dx = rd.x; world.dy = rd.y; world.dz = rd.z;
        if (direct) identity_space(world, ro, rd);
        setup_space(world);
        SpaceRay r = world;
        bool bottom = direct;
        int cur_inst = direct ? (p.roots ? 0 : p.direct_inst) : -1;
        float tlimit = best_t * IMBART_SLACK;

        uint2 stack[kStackSize];
        int sp = 0;
        // Root group: one internal child in slot 0.
        uint32_t g_base = (uint32_t)(p.roots ? (root_word & ~kDirectRootBit) : direct ? p.direct_root : p.root),
                 g_imask = 1u, g_hits = 1u << (0u ^ r.oct);
        uint32_t t_base = 0, t_mask = 0;
        bool done = false;

        while (!done) {
            if (t_mask == 0 && g_hits != 0) {
                const uint32_t bitpos = __ffs(g_hits) - 1;
                g_hits &= g_hits - 1;
                const uint32_t slot = bitpos ^ r.oct;
                const uint32_t idx = g_base + __popc(g_imask & ((1u << slot) - 1u));
                if (g_hits != 0) {
                    if (sp == kStackSize) { atomicAdd(p.error_flags, 1); break; }
                    stack[sp++] = make_uint2(g_base | (kEntryNode << kTypeShift), (g_hits << 8) | g_imask);
                }
                intersect_node<8, !kAnyHit>(p.nodes + idx, r, tmin, tlimit, g_base, g_imask, g_hits, t_base, t_mask);
                if (kStats) st.nodes++;
            }

            if (t_mask != 0) {
                if (bottom) {
                    while (t_mask != 0) {
                        const uint32_t i = __ffs(t_mask) - 1;
                        t_mask &= t_mask - 1;
                        const float4* tp = reinterpret_cast<const float4*>(p.tris + t_base + i);
                        const float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
                        if (kStats) st.tris++;
                        float t, u, v;
                        if (!tri_test(r, a, b, c, t, u, v)) continue;
                        if (!(t >= tmin)) continue;
                        const int tri = __float_as_int(a.w);
                        const bool closer = (t < best_t) ||
                            (t == best_t && (best_tri < 0 || cur_inst < best_inst ||
                                             (cur_inst == best_inst && tri < best_tri)));
                        if (!closer) continue;
                        if (kMasked && !mask_opaque(p, tri, u, v)) continue;
                        best_t = t; best_u = u; best_v = v; best_tri = tri; best_inst = cur_inst;
                        tlimit = best_t * IMBART_SLACK;
                        if (kAnyHit) { done = true; break; }
                    }
                    if (done) break;
                } else {
                    // Enter the next instance of the group.
                    const uint32_t i = __ffs(t_mask) - 1;
                    t_mask &= t_mask - 1;
                    if (sp + 3 > kStackSize) { atomicAdd(p.error_flags, 1); break; }
                    if (g_hits != 0)
                        stack[sp++] = make_uint2(g_base | (kEntryNode << kTypeShift), (g_hits << 8) | g_imask);
                    if (t_mask != 0)
                        stack[sp++] = make_uint2(t_base | (kEntryInst << kTypeShift), t_mask);
                    stack[sp++] = make_uint2(kEntryMarker << kTypeShift, 0u);
                    t_mask = 0;
                    const float4* ip = reinterpret_cast<const float4*>(p.insts + t_base + i);
                    const float4 m0 = __ldg(ip + 0), m1 = __ldg(ip + 1), m2 = __ldg(ip + 2);
                    const int4 meta = __ldg(reinterpret_cast<const int4*>(ip + 3));
                    if (kStats) st.insts++;
                    r.ox = xform_row(m0, world.ox, world.oy, world.oz, 1.0f);
                    r.oy = xform_row(m1, world.ox, world.oy, world.oz, 1.0f);
                    r.oz = xform_row(m2, world.ox, world.oy, world.oz, 1.0f);
                    r.dx = xform_row(m0, world.dx, world.dy, world.dz, 0.0f);
                    r.dy = xform_row(m1, world.dx, world.dy, world.dz, 0.0f);
                    r.dz = xform_row(m2, world.dx, world.dy, world.dz, 0.0f);
                    setup_space(r);
                    cur_inst = meta.x;
                    bottom = true;
                    g_base = (uint32_t)meta.y; g_imask = 1u; g_hits = 1u << (0u ^ r.oct);
                    continue;
                }
            }

            if (g_hits == 0 && t_mask == 0) {
                // Pop the next group.
                for (;;) {
                    if (sp == 0) { done = true; break; }
                    const uint2 e = stack[--sp];
                    const uint32_t type = e.x >> kTypeShift;
                    if (type == kEntryMarker) {
                        r = world; bottom = false; cur_inst = -1;
                        continue;
                    }
                    if (type == kEntryInst) { t_base = e.x & kIndexMask; t_mask = e.y; break; }
                    g_base = e.x & kIndexMask; g_imask = e.y & 0xffu; g_hits = e.y >> 8;
                    break;
                }
            }
        }
    }

    int4 h;
    h.x = best_tri;
    h.y = best_tri >= 0 ? best_inst : -1;
    h.z = __float_as_int(best_t);
    h.w = __float_as_int(best_tri >= 0 ? best_u : 0.0f);
    p.hits[ray_index] = h;
    if (p.v_out) p.v_out[ray_index] = best_tri >= 0 ? best_v : 0.0f;
}

// ---------------------------------------------------------------------------------------
// Persistent-warp traversal.
//
// Each warp keeps 32 rays in flight and pulls new ray indices from a global counter with one
// warp-aggregated atomic whenever `refill_lanes` of its lanes have finished, so lanes do not
// idle until the slowest ray of a static batch ends. The loop follows the node-group /
// triangle-group scheme of Ylitie, Karras and Laine (HPG 2017): a node step pops the next hit
// child of the current group and intersects its 8 boxes, producing a group of hit internal
// children and a group of hit leaf primitives. The stack lives in shared memory (kSh entries
// per thread, laid out so that neighbouring threads touch neighbouring words) and spills to
// local memory. Results are identical to the per-thread kernel: same tests, same tie rule.
//
// Triangle groups are tested in one of two ways:
//  * per lane (kCoop false): a lane tests up to `tri_batch` triangles of its group per loop
//    trip (the rest wait for the next trip while lanes with node work take their node step);
//    triangle tests are postponed (the group goes onto the stack) while fewer than
//    postpone_lanes/32 of the live lanes would test triangles together;
//  * cooperatively (kCoop true): after the node step, the warp lists every (ray, triangle)
//    pair its lanes' triangle groups hold and all 32 lanes — idle and finished ones included —
//    test 32 pairs per pass, reading the owning lane's ray through shuffles and loading the
//    pair's triangle itself (staging a pass's triangles in shared memory with coalesced warp
//    loads measured slower: the records hit in L1/L2, and the buffer's shared memory is worth
//    more as L1). Each owner's closest candidate is found by shared-memory atomic minima over
//    (t, triangle id), any-hit queries take the first accepted pair in the group's test
//    order, so hits and the work counters equal those of the per-lane tests.
// ---------------------------------------------------------------------------------------
template <bool kAnyHit, bool kMasked, bool kStats, int kBlock, int kMinBlocks, int kSh, bool kCoop, int kSlots = 8,
          bool kFlat = false>
__global__ void __launch_bounds__(kBlock, kMinBlocks) trace_persistent(TraceParams p) {
    constexpr unsigned kFull = 0xffffffffu;
    constexpr uint32_t kOct = kSlots - 1;             // octant bits that order a node's slots
    // kFlat: the launch's scene is one identity instance (p.direct_root >= 0, no per-ray
    // roots); every ray starts in its tree and never leaves it, so the instance entry and
    // exit, the saved world ray and the current-instance register are compiled out.
    constexpr int kCW = kCoop ? kBlock / 32 : 1;     // warps with cooperative-phase slots
    __shared__ uint2 sstack[kSh][kBlock];
    __shared__ uint32_t s_key[kCW][32];              // per owner lane: smallest key of a pass
    __shared__ int s_tri[kCW][32];                   // per owner lane: its winning triangle id
    __shared__ float4 s_hit[kCW][32];                // per owner lane: the winner's t, u, v
    // The world ray (origin, direction, inverse direction, pad, octant): instance entries read
    // the world direction from here, exits restore the rest. Shared memory rather than
    // registers (11 registers fewer; measured +4-6 % on the instanced scene's ray sets); the
    // direction is not needed in registers after the ray's set-up. Flat kernels never leave
    // the tree.
    __shared__ float s_world[kFlat ? 1 : 11][kFlat ? 1 : kBlock];
    // The best hit's u and v (read once, when the ray finishes): shared memory, not registers
    // (+0.5-1 % on both scenes' ray sets; the 64-register shapes then spill 8 bytes, not 60-130).
    __shared__ float s_uv[2][kBlock];
    uint2 lstack[kStackSize - kSh];
    const int tid = threadIdx.x;
    const unsigned lane = tid & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;

    int ray = -1;                       // -1: idle (wants a ray), >= count: queue exhausted
    SpaceRay r;                         // current space (world or instance)
    float tmin = 0.0f, best_t = 0.0f, tlimit = 0.0f;
    int best_tri = -1, best_inst = -1, cur_inst = -1;
    bool bottom = false;
    uint32_t g_base = 0, g_imask = 0, g_hits = 0, t_base = 0, t_mask = 0;
    int sp = 0;
    RayStats st;
    r.ox = r.oy = r.oz = 0.0f;
    r.Sx = r.Sy = r.Sz = 0.0f;
    r.kx = r.ky = r.kz = 0;
    const int count = p.count_ptr ? min(__ldg(p.count_ptr), p.count) : p.count;

    auto push = [&](uint32_t x, uint32_t y) -> bool {
        if (sp >= kStackSize) return false;
        if (sp < kSh) sstack[sp][tid] = make_uint2(x, y);
        else lstack[sp - kSh] = make_uint2(x, y);
        ++sp;
        return true;
    };
    auto finish = [&]() {
        int4 h;
        h.x = best_tri;
        h.y = best_tri >= 0 ? (kFlat ? p.direct_inst : best_inst) : -1;
        h.z = __float_as_int(best_t);
        h.w = __float_as_int(best_tri >= 0 ? s_uv[0][tid] : 0.0f);
        p.hits[ray] = h;
        if (p.v_out) p.v_out[ray] = best_tri >= 0 ? s_uv[1][tid] : 0.0f;
        ray = -1;
    };

    for (;;) {
        // Refill idle lanes in warp-wide batches.
        const unsigned idle = __ballot_sync(kFull, ray < 0);
        unsigned live = __ballot_sync(kFull, ray >= 0 && ray < count);
        if (idle != 0u && (live == 0u || __popc(idle) >= p.refill_lanes)) {
            const int leader = __ffs(idle) - 1;
            int base = 0;
            if ((int)lane == leader) base = atomicAdd(p.work, __popc(idle));
            base = __shfl_sync(kFull, base, leader);
            if (ray < 0) {
                const int idx = base + __popc(idle & lt_mask);
                if (idx >= count) {
                    ray = count;
                } else {
                    ray = idx;
                    const float4 ro = __ldg(p.rays + 2 * ray + 0);
                    const float4 rd = __ldg(p.rays + 2 * ray + 1);
                    tmin = ro.w; best_t = rd.w;
                    best_tri = -1; best_inst = -1; cur_inst = -1; bottom = false; sp = 0;
                    if (!((tmin <= best_t) && (rd.x != 0.0f || rd.y != 0.0f || rd.z != 0.0f))) {
                        finish();
                    } else {
                        const int root_word = (!kFlat && p.roots) ? __ldg(p.roots + ray) : p.root;
                        const bool direct = kFlat || (p.roots ? (root_word & kDirectRootBit) != 0 : p.direct_root >= 0);
                        r.ox = ro.x; r.oy = ro.y; r.oz = ro.z;
                        r.dx = rd.x; r.dy = rd.y; r.dz = rd.z;
                        if (direct) {
                            identity_space(r, ro, rd);
                            bottom = true;
                            cur_inst = (!kFlat && p.roots) ? 0 : p.direct_inst;
                        }
                        setup_space(r);
                        if (!kFlat) {
                            s_world[0][tid] = r.ox; s_world[1][tid] = r.oy; s_world[2][tid] = r.oz;
                            s_world[3][tid] = r.dx; s_world[4][tid] = r.dy; s_world[5][tid] = r.dz;
                            s_world[6][tid] = r.ix; s_world[7][tid] = r.iy; s_world[8][tid] = r.iz;
                            s_world[9][tid] = r.pad; s_world[10][tid] = __uint_as_float(r.oct);
                        }
                        tlimit = best_t * IMBART_SLACK;
                        g_base = (uint32_t)((!kFlat && p.roots) ? (root_word & ~kDirectRootBit)
                                                                : direct ? p.direct_root : p.root);
                        g_imask = 1u; g_hits = 1u << (0u ^ (r.oct & kOct));
                        t_mask = 0;
                    }
                }
            }
            live = __ballot_sync(kFull, ray >= 0 && ray < count);
        }
        if (live == 0u) {
            if (__ballot_sync(kFull, ray < 0) == 0u) break;   // every lane exhausted
            continue;
        }
        const bool active = ray >= 0 && ray < count;
        // The per-lane form lets idle lanes skip the trip; the cooperative form keeps every
        // lane for the triangle phase.
        if (!kCoop && !active) continue;
        const int n_live = __popc(live);
        bool next = !active;   // this lane's trip is over (finished, or entered an instance)

        // Node step.
        if (!next && t_mask == 0 && g_hits != 0) {
            const uint32_t bitpos = __ffs(g_hits) - 1;
            g_hits &= g_hits - 1;
            const uint32_t slot = bitpos ^ (r.oct & kOct);
            const uint32_t idx = g_base + __popc(g_imask & ((1u << slot) - 1u));
            if (g_hits != 0 && !push(g_base | (kEntryNode << kTypeShift), (g_hits << 8) | g_imask)) {
                atomicAdd(p.error_flags, 1);
                finish();
                next = true;
            } else {
                intersect_node<kSlots, !kAnyHit>(p.nodes + idx, r, tmin, tlimit, g_base, g_imask, g_hits, t_base, t_mask);
                if (kStats) st.nodes++;
            }
        }

        // Primitive step: instance entry, and per-lane triangle tests.
        if (!next && t_mask != 0) {
            if (kFlat || bottom) {
                if (!kCoop) {
                    bool stop = false;
                    int tested = 0;
                    while (t_mask != 0) {
                        // The rest of the group waits for the next trip (the lanes with node
                        // work take their node step meanwhile).
                        if (p.tri_batch > 0 && tested == p.tri_batch) break;
                        ++tested;
                        // Postpone only while node work remains, so that a ray with nothing
                        // but triangles left always makes progress.
                        if (g_hits != 0 && __popc(__activemask()) * 32 < n_live * p.postpone_lanes) {
                            if (!push(t_base | (kEntryTri << kTypeShift), t_mask)) {
                                atomicAdd(p.error_flags, 1);
                                stop = true;
                            }
                            t_mask = 0;
                            break;
                        }
                        const uint32_t i = __ffs(t_mask) - 1;
                        t_mask &= t_mask - 1;
                        const float4* tp = reinterpret_cast<const float4*>(p.tris + t_base + i);
                        const float4 a = __ldg(tp + 0), b = __ldg(tp + 1), c = __ldg(tp + 2);
                        if (kStats) st.tris++;
                        float t, u, v;
                        if (!tri_test(r, a, b, c, t, u, v)) continue;
                        if (!(t >= tmin)) continue;
                        const int tri = __float_as_int(a.w);
                        const bool closer = (t < best_t) ||
                            (t == best_t && (kFlat ? (best_tri < 0 || tri < best_tri)
                                                   : (best_tri < 0 || cur_inst < best_inst ||
                                                      (cur_inst == best_inst && tri < best_tri))));
                        if (!closer) continue;
                        if (kMasked && !mask_opaque(p, tri, u, v)) continue;
                        best_t = t; s_uv[0][tid] = u; s_uv[1][tid] = v; best_tri = tri; best_inst = cur_inst;
                        tlimit = best_t * IMBART_SLACK;
                        if (kAnyHit) { stop = true; break; }
                    }
                    if (stop) { finish(); next = true; }
                }
            } else {
                // Enter the next instance of the group.
                const uint32_t i = __ffs(t_mask) - 1;
                t_mask &= t_mask - 1;
                bool ok = true;
                if (g_hits != 0) ok = push(g_base | (kEntryNode << kTypeShift), (g_hits << 8) | g_imask);
                if (ok && t_mask != 0) ok = push(t_base | (kEntryInst << kTypeShift), t_mask);
                if (ok) ok = push(kEntryMarker << kTypeShift, 0u);
                if (!ok) {
                    atomicAdd(p.error_flags, 1);
                    finish();
                } else {
                    t_mask = 0;
                    const float4* ip = reinterpret_cast<const float4*>(p.insts + t_base + i);
                    const float4 m0 = __ldg(ip + 0), m1 = __ldg(ip + 1), m2 = __ldg(ip + 2);
                    const int4 meta = __ldg(reinterpret_cast<const int4*>(ip + 3));
                    if (kStats) st.insts++;
                    const float wx = r.ox, wy = r.oy, wz = r.oz;
                    const float vx = s_world[3][tid], vy = s_world[4][tid], vz = s_world[5][tid];
                    r.ox = xform_row(m0, wx, wy, wz, 1.0f);
                    r.oy = xform_row(m1, wx, wy, wz, 1.0f);
                    r.oz = xform_row(m2, wx, wy, wz, 1.0f);
                    r.dx = xform_row(m0, vx, vy, vz, 0.0f);
                    r.dy = xform_row(m1, vx, vy, vz, 0.0f);
                    r.dz = xform_row(m2, vx, vy, vz, 0.0f);
                    setup_space(r);
                    cur_inst = meta.x;
                    bottom = true;
                    g_base = (uint32_t)meta.y; g_imask = 1u; g_hits = 1u << (0u ^ (r.oct & kOct));
                }
                next = true;
            }
        }

        // Cooperative triangle phase (every lane of the warp takes part).
        if (kCoop) {
            const bool want = !next && (kFlat || bottom) && t_mask != 0;
            if (__ballot_sync(kFull, want) != 0u) {
                const int w = tid >> 5;
                const int cnt = want ? __popc(t_mask) : 0;
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(kFull, incl, o);
                    if ((int)lane >= o) incl += y;
                }
                const int total = __shfl_sync(kFull, incl, 31);
                const int excl = incl - cnt;
                const uint32_t kpack = (uint32_t)r.kx | ((uint32_t)r.ky << 2) | ((uint32_t)r.kz << 4);
                int found_k = -1;    // any hit: position of the group's first accepted triangle
                for (int pass = 0; pass < total; pass += 32) {
                    const int j = pass + (int)lane;
                    // Owner of pair j: the first lane whose inclusive count exceeds j.
                    int o = 0;
#pragma unroll
                    for (int step = 16; step >= 1; step >>= 1) {
                        const int c = __shfl_sync(kFull, incl, o + step - 1);
                        if (c <= j) o += step;
                    }
                    const int o_excl = __shfl_sync(kFull, excl, o);
                    const uint32_t o_mask = __shfl_sync(kFull, t_mask, o);
                    const uint32_t o_base = __shfl_sync(kFull, t_base, o);
                    SpaceRay q;
                    q.ox = __shfl_sync(kFull, r.ox, o);
                    q.oy = __shfl_sync(kFull, r.oy, o);
                    q.oz = __shfl_sync(kFull, r.oz, o);
                    q.Sx = __shfl_sync(kFull, r.Sx, o);
                    q.Sy = __shfl_sync(kFull, r.Sy, o);
                    q.Sz = __shfl_sync(kFull, r.Sz, o);
                    const uint32_t qk = __shfl_sync(kFull, kpack, o);
                    q.kx = (int)(qk & 3u); q.ky = (int)((qk >> 2) & 3u); q.kz = (int)((qk >> 4) & 3u);
                    const float o_tmin = __shfl_sync(kFull, tmin, o);
                    const float o_best = __shfl_sync(kFull, best_t, o);
                    const bool has = j < total;
                    const int k = j - o_excl;
                    const int ti = has ? (int)(o_base + nth_set_bit(o_mask, k)) : -1;
                    float4 a, b, c;
                    if (has) {
                        const float4* tp = reinterpret_cast<const float4*>(p.tris + ti);
                        a = __ldg(tp + 0); b = __ldg(tp + 1); c = __ldg(tp + 2);
                    }
                    bool cand = false;
                    float t = 0.0f, u = 0.0f, v = 0.0f;
                    int tri = 0;
                    if (has && tri_test(q, a, b, c, t, u, v) && t >= o_tmin && t <= o_best) {
                        tri = __float_as_int(a.w);
                        cand = !kMasked || mask_opaque(p, tri, u, v);
                    }
                    const bool in_pass = want && excl < pass + 32 && incl > pass;
                    if (in_pass) { s_key[w][lane] = 0xffffffffu; s_tri[w][lane] = 0x7fffffff; }
                    __syncwarp();
                    uint32_t key;
                    if (kAnyHit) {
                        key = (uint32_t)k;            // the group's test order
                    } else {
                        // t as an ordered unsigned key (+0 and -0 equal, as the tie rule has it)
                        const uint32_t tb = __float_as_uint(__fadd_rn(t, 0.0f));
                        key = (tb & 0x80000000u) ? ~tb : (tb | 0x80000000u);
                    }
                    if (cand) atomicMin(&s_key[w][o], key);
                    __syncwarp();
                    bool win = cand && s_key[w][o] == key;
                    if (!kAnyHit) {
                        if (win) atomicMin(&s_tri[w][o], tri);
                        __syncwarp();
                        win = win && s_tri[w][o] == tri;
                    }
                    if (win) {
                        if (kAnyHit) s_tri[w][o] = tri;
                        s_hit[w][o] = make_float4(t, u, v, 0.0f);
                    }
                    __syncwarp();
                    if (in_pass && s_key[w][lane] != 0xffffffffu) {
                        const int tc = s_tri[w][lane];
                        const float4 hv = s_hit[w][lane];
                        if (kAnyHit) {
                            if (found_k < 0) {
                                found_k = (int)s_key[w][lane];
                                best_t = hv.x; s_uv[0][tid] = hv.y; s_uv[1][tid] = hv.z; best_tri = tc; best_inst = cur_inst;
                            }
                        } else {
                            const bool closer = (hv.x < best_t) ||
                                (hv.x == best_t && (kFlat ? (best_tri < 0 || tc < best_tri)
                                                          : (best_tri < 0 || cur_inst < best_inst ||
                                                             (cur_inst == best_inst && tc < best_tri))));
                            if (closer) {
                                best_t = hv.x; s_uv[0][tid] = hv.y; s_uv[1][tid] = hv.z; best_tri = tc; best_inst = cur_inst;
                                tlimit = best_t * IMBART_SLACK;
                            }
                        }
                    }
                    __syncwarp();
                }
                if (want) {
                    if (kStats) st.tris += (kAnyHit && found_k >= 0) ? (uint32_t)(found_k + 1) : (uint32_t)cnt;
                    t_mask = 0;
                    if (kAnyHit && found_k >= 0) { finish(); next = true; }
                }
            }
        }

        // Pop the next group when the current ones are exhausted.
        if (!next && ray >= 0 && g_hits == 0 && t_mask == 0) {
            for (;;) {
                if (sp == 0) { finish(); break; }
                --sp;
                const uint2 e = sp < kSh ? sstack[sp][tid] : lstack[sp - kSh];
                const uint32_t type = e.x >> kTypeShift;
                if (!kFlat && type == kEntryMarker) {
                    r.ox = s_world[0][tid]; r.oy = s_world[1][tid]; r.oz = s_world[2][tid];
                    r.ix = s_world[6][tid]; r.iy = s_world[7][tid]; r.iz = s_world[8][tid];
                    r.pad = s_world[9][tid]; r.oct = __float_as_uint(s_world[10][tid]);
                    bottom = false; cur_inst = -1;
                    continue;
                }
                if (type == kEntryNode) { g_base = e.x & kIndexMask; g_imask = e.y & 0xffu; g_hits = e.y >> 8; }
                else { t_base = e.x & kIndexMask; t_mask = e.y; }
                break;
            }
        }
    }

    if (kStats) {
        const unsigned n = __reduce_add_sync(kFull, st.nodes);
        const unsigned t = __reduce_add_sync(kFull, st.tris);
        const unsigned k = __reduce_add_sync(kFull, st.insts);
        if (lane == 0) {
            atomicAdd(p.stats + 0, (unsigned long long)n);
            atomicAdd(p.stats + 1, (unsigned long long)t);
            atomicAdd(p.stats + 2, (unsigned long long)k);
        }
    }
    // The last warp to finish resets the work counter for the next launch on this slot.
    if (lane == 0) {
        __threadfence();
        if (atomicAdd(p.work + 1, 1) == p.total_warps - 1) {
            atomicExch(p.work + 0, 0);
            atomicExch(p.work + 1, 0);
        }
    }
}

template <bool kAnyHit, bool kMasked, bool kStats>
__global__ void __launch_bounds__(128) trace_kernel(TraceParams p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    RayStats st;
    const int count = p.count_ptr ? min(__ldg(p.count_ptr), p.count) : p.count;
    if (i < count) trace_one<kAnyHit, kMasked, kStats>(p, i, st);
    if (kStats) {
        // Warp-aggregated accumulation of the per-ray counters.
        const unsigned m = __activemask();
        const unsigned n = __reduce_add_sync(m, st.nodes);
        const unsigned t = __reduce_add_sync(m, st.tris);
        const unsigned k = __reduce_add_sync(m, st.insts);
        if ((threadIdx.x & 31) == __ffs(m) - 1) {
            atomicAdd(p.stats + 0, (unsigned long long)n);
            atomicAdd(p.stats + 1, (unsigned long long)t);
            atomicAdd(p.stats + 2, (unsigned long long)k);
        }
    }
}

}  // namespace imbart
