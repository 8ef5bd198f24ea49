/*
 * traversal_gpu.h — drop-in replacement for the header of the external AnyDSL/traversal GPU
 * library, which the reference includes inside a namespace
 * (src/imbatracer/core/traversal_interface.h:8-10):
 *
 *     namespace traversal_gpu {
 *     #include <traversal_gpu.h>
 *     }
 *
 * It therefore includes nothing and only declares the types and the two entry points, with
 * C linkage so that the namespaced declarations bind to libimbart's unmangled symbols.
 * Layouts are identical to the imbart_* types of imbart.h. Entry points: see imbart.h
 * (intersect_gpu_masked_instanced / occluded_gpu_masked_instanced, device pointers).
 */
#ifndef IMBART_TRAVERSAL_GPU_H
#define IMBART_TRAVERSAL_GPU_H

struct Vec4 { float x, y, z, w; };
struct Vec2 { float x, y; };
struct Ray { Vec4 org; Vec4 dir; };
struct Hit { int tri_id; int inst_id; float tmax; float u; };
struct BBox { float lo_x, hi_x, lo_y, hi_y, lo_z, hi_z; };
struct Node { BBox left_bb; BBox right_bb; int left; int right; int pad[2]; };
struct InstanceNode { float transf[12]; int id; int next; int pad[2]; };
struct TransparencyMask { int width; int height; int offset; };

#ifdef __cplusplus
extern "C" {
#endif
void intersect_gpu_masked_instanced(int root, Node* nodes, InstanceNode* instances, Vec4* tris, Ray* rays,
                                    Hit* hits, int* indices, Vec2* texcoords, TransparencyMask* masks,
                                    char* mask_buffer, int count);
void occluded_gpu_masked_instanced(int root, Node* nodes, InstanceNode* instances, Vec4* tris, Ray* rays,
                                   Hit* hits, int* indices, Vec2* texcoords, TransparencyMask* masks,
                                   char* mask_buffer, int count);
#ifdef __cplusplus
}
#endif

#endif
