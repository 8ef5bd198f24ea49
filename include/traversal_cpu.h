/*
 * traversal_cpu.h — drop-in replacement for the header of the external AnyDSL/traversal CPU
 * library, which the reference includes inside a namespace
 * (src/imbatracer/core/traversal_interface.h:4-6):
 *
 *     namespace traversal_cpu {
 *     #include <traversal_cpu.h>
 *     }
 *
 * Declares the types of the four-wide CPU layout (cpu_adapter.cpp:56-208) and the two
 * entry points with C linkage. In libimbart these take HOST pointers and run on the GPU
 * (the scene is converted once and kept resident; rays/hits are copied per call).
 */
#ifndef IMBART_TRAVERSAL_CPU_H
#define IMBART_TRAVERSAL_CPU_H

struct Vec4 { float x, y, z, w; };
struct Vec2 { float x, y; };
struct Ray { Vec4 org; Vec4 dir; };
struct Hit { int tri_id; int inst_id; float tmax; float u; };
struct Node {
    float min_x[4], max_x[4], min_y[4], max_y[4], min_z[4], max_z[4];
    int children[4];
};
struct InstanceNode { float transf[12]; int id; int next; int pad[2]; };
struct TransparencyMask { int width; int height; int offset; };

#ifdef __cplusplus
extern "C" {
#endif
void intersect_cpu_masked_instanced(int root, Node* nodes, InstanceNode* instances, Vec4* tris, Ray* rays,
                                    Hit* hits, int* indices, Vec2* texcoords, TransparencyMask* masks,
                                    char* mask_buffer, int count);
void occluded_cpu_masked_instanced(int root, Node* nodes, InstanceNode* instances, Vec4* tris, Ray* rays,
                                   Hit* hits, int* indices, Vec2* texcoords, TransparencyMask* masks,
                                   char* mask_buffer, int count);
#ifdef __cplusplus
}
#endif

#endif
