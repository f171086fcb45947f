// Device-resident scene: triangles in BVH leaf order, the BVH, per-face
// tables, coplanar face groups and the selected diffraction edges.
#pragma once

#include "common.cuh"
#include "utd.cuh"

namespace wcb {

constexpr int kStackDepth = 64;  // per-thread traversal stack entries (shared memory)

// compile tolerances (shared by the host compile and the device refit)
constexpr double kPlaneGroupQuant = 1.0e-4;  // propagation/geometry.py:113
constexpr double kEdgePlaneTol = 1.34e-5;    // propagation/geometry.py:37
constexpr double kEndpointQuant = 1.0e-4;    // scene/resources.py:296
constexpr double kNormalCosTol = 1.0 - 1.0e-5;
constexpr double kPlaneTolerance = 1.0e-3;   // rayd/reflection.cpp:50

// BVH node: both child boxes plus the child references (64 bytes, four
// 16-byte loads).  child >= 0: internal node; child < 0: leaf ~slot.
struct __align__(16) BvhNode {
    float4 a;  // c0.lo.xyz, c0.hi.x
    float4 b;  // c0.hi.yz, c1.lo.xy
    float4 c;  // c1.lo.z, c1.hi.xyz
    int4 d;    // left, right, -, -
};

struct SceneDev {
    int num_vertices;
    int num_faces;
    int num_groups;
    int num_edges;        // selected edges
    int root;             // root child reference (internal node index, or ~slot, or INT_MIN when empty)
    int max_depth;        // BVH depth (root = 0)
    int stack_entries;    // traversal stack entries per thread (BVH depth + 2, at most kStackDepth)
    // geometry
    const float* vertices;     // (V,3)
    const int* faces;          // (F,3)
    const float4* tri;         // (F*3) leaf order: v0|face, v1|group, v2|pad
    const BvhNode* nodes;      // (F-1)
    // per face (original order)
    const float* face_normal;  // (F,3) unit, fp32
    const double* face_plane;  // (F,4) unit normal + offset n.v0, fp64
    const int* face_group;     // (F)
    const int* face_material;  // (F)
    // groups
    const int* group_rep;          // (G)
    const int* group_member_off;   // (G+1)
    const int* group_members;      // (F) ascending face index within a group
    const double* group_plane;     // (G,4) representative normal + offset (anchor = rep's v0)
    const float* group_box;        // (G,6) lo.xyz hi.xyz padded by the plane tolerance
    // edges
    const EdgeDev* edges;          // (E)
    double diagonal;               // scene bounding-box diagonal
};

}  // namespace wcb
