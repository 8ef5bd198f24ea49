/*
 * Types shared by the oracle's C sources. TEST INFRASTRUCTURE ONLY: the oracle is the CPU
 * restatement that checks libimbart; nothing in the product imports, links or runs it.
 *
 * Layouts are the reference boundary's (see include/imbart.h for the field meanings):
 * rays {org.xyz, tmin; dir.xyz, tmax}, hits {tri_id, inst_id, tmax, u}, two-wide GPU nodes
 * (gpu_adapter.cpp:84-101), 3-Vec4 triangles with the id in v1.w and the run sentinel
 * 0x80000000 in the last v2.w (gpu_adapter.cpp:129-141), 64-byte instance nodes
 * (cpu_adapter.cpp:346-365).
 */
#ifndef ORACLE_TYPES_H
#define ORACLE_TYPES_H

#include <stdint.h>

typedef struct { float x, y, z, w; } o_vec4;
typedef struct { float x, y; } o_vec2;
typedef struct { o_vec4 org, dir; } o_ray;
typedef struct { int tri_id, inst_id; float tmax, u; } o_hit;
typedef struct { float lo_x, hi_x, lo_y, hi_y, lo_z, hi_z; } o_bbox;
typedef struct { o_bbox left_bb, right_bb; int left, right, pad[2]; } o_node2;
typedef struct { float transf[12]; int id, next, pad[2]; } o_inst;
typedef struct { int width, height, offset; } o_mask;

/* The compressed 8-wide layout of libimbart, mirrored for byte accounting. */
typedef struct {
    float px, py, pz;
    uint8_t ex, ey, ez, imask;
    uint32_t child_base, prim_base;
    uint8_t meta[8];
    uint8_t qlo_x[8], qhi_x[8], qlo_y[8], qhi_y[8], qlo_z[8], qhi_z[8];
} o_wnode;
typedef struct { float v0[3]; int32_t id; float v1[3]; int32_t p0; float v2[3]; int32_t p1; } o_wtri;
typedef struct { float m[12]; int32_t id, root, pad[2]; } o_winst;

#endif
