// qbvh.h -- memory layout of the 4-wide bounding volume hierarchy shared by the host builder and
// the sm_100a traversal kernels.
//
// The reference keeps one Lass QbvhTree<Triangle, ..., SAHSplitHeuristics> per TriangleMesh
// (src/liar/scenery/triangle_mesh.h:53) and calls its intersect / intersects from
// TriangleMesh::doIntersect / doIsIntersecting (src/liar/scenery/triangle_mesh.cpp:291-330).
// Lass is not part of the reference sources, so the tree here is an own design:
//
//   QNode (128 B, one L2 line): the four child boxes as structure-of-arrays float4 rows so
//   that one thread reads all four boxes with six 16-byte loads, plus the child links.
//     child[c] >= 0 : index of an inner QNode
//     child[c] <  0 : leaf, packed as 0x80000000 | count << 27 | first, holding the triangles
//                     tris[first .. first + count) (count <= 8, first < 2^27); count 0 marks an
//                     empty slot, whose box is also inverted so that it never hits
//     count[c]      : the leaf's triangle count again (0 for inner nodes), kept for tools
//
//   QTri (48 B): v0, e1 = v1 - v0, e2 = v2 - v0 as three float4, the original triangle index in
//   the w lane of the first; e1.w = 0. A sphere primitive has its centre in v0, its radius in
//   e1.x and e1.w = 1. e1/e2 are the same IEEE single subtractions that the
//   Moller-Trumbore test performs, so precomputing them changes no bit of the result.
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __CUDACC__
#define LIAR_HD __host__ __device__
#else
#define LIAR_HD
#endif

namespace liar_gpu {

struct alignas(16) F4 { float x, y, z, w; };
struct alignas(16) I4 { int32_t x, y, z, w; };

struct alignas(128) QNode {
    F4 lo_x, hi_x, lo_y, hi_y, lo_z, hi_z;  // child c bounds in lane c
    I4 child;                               // see above
    I4 count;                               // leaf triangle count per child, 0 for inner/empty
};
static_assert(sizeof(QNode) == 128, "QNode must be one 128-byte line");
// the traversal selects a child row's near or far plane by these offsets (hi_* = lo_* + 16 bytes)
static_assert(offsetof(QNode, lo_x) == 0 && offsetof(QNode, hi_x) == 16 && offsetof(QNode, lo_y) == 32 &&
                  offsetof(QNode, hi_y) == 48 && offsetof(QNode, lo_z) == 64 && offsetof(QNode, hi_z) == 80,
              "QNode plane rows");

struct alignas(16) QTri {
    F4 v0;   // v0.xyz, w = original triangle index (int bits)
    F4 e1;   // v1 - v0, w = 0
    F4 e2;   // v2 - v0, w = 0
};
static_assert(sizeof(QTri) == 48, "QTri must be 48 bytes");

// Build output in host memory.
struct QBVHHost {
    QNode* nodes = nullptr;
    uint64_t n_nodes = 0;
    QTri* tris = nullptr;
    uint64_t n_tris = 0;
    uint64_t n_leaves = 0;
    uint32_t max_depth = 0;
    uint32_t stack_needed = 0;
    double sah_cost = 0.0;
    // set when the whole mesh is a single leaf below a root with one child
};

struct BuildOptions {
    int max_leaf_size = 4;
    int sah_bins = 32;
    float traversal_cost = 1.0f;
    int threads = 0;
};

// Builds the tree; returns 0 on success, a negative LIAR_ERR_* otherwise (msg filled).
int build_qbvh(const float* vertices, uint64_t n_vertices, const uint32_t* triangles, uint64_t n_triangles,
               const BuildOptions& opts, QBVHHost& out, char* msg, size_t msg_len);
// The same over triangles and spheres (n_spheres x 4: centre, radius); sphere k is primitive
// n_triangles + k, its QTri holding the centre in v0, the radius in e1.x and 1 in e1.w
int build_qbvh(const float* vertices, uint64_t n_vertices, const uint32_t* triangles, uint64_t n_triangles,
               const float* spheres, uint64_t n_spheres, const BuildOptions& opts, QBVHHost& out, char* msg,
               size_t msg_len);
void free_qbvh(QBVHHost& q);

}  // namespace liar_gpu
