// tri_exact.h -- the ray/triangle test shared, operation for operation, by the CUDA kernels and
// the C++ host code.
//
// The reference calls Lass's TriangleMesh3D::intersectFilter (src/liar/scenery/triangle_mesh.cpp:301),
// whose source is not part of the reference. The test restated here is the published
// Moller & Trumbore 1997 algorithm ("Fast, minimum storage ray/triangle intersection"), two-sided
// (no back-face culling, like the reference's meshes which report both seEntering and
// seLeaving hits, triangle_mesh.cpp:303-308).
//
// Every operation is an explicitly rounded IEEE single-precision add, subtract, multiply or
// reciprocal, evaluated in a fixed order, with no fused multiply-add. A C++ build compiled
// with -ffp-contract=off and without -ffast-math performs the very same roundings, so the
// t, u and v of a given (ray, triangle) pair are bit-identical on the CPU and on the GPU.
#pragma once

#ifdef __CUDACC__
#define TX_HD __host__ __device__ __forceinline__
#else
#define TX_HD inline
#endif
#ifdef __CUDA_ARCH__
#define TX_ADD(a, b) __fadd_rn((a), (b))
#define TX_SUB(a, b) __fsub_rn((a), (b))
#define TX_MUL(a, b) __fmul_rn((a), (b))
#define TX_RCP(a) __frcp_rn(a)
#define TX_DIV(a, b) __fdiv_rn((a), (b))
#define TX_SQRT(a) __fsqrt_rn(a)
#else
#define TX_ADD(a, b) ((a) + (b))
#define TX_SUB(a, b) ((a) - (b))
#define TX_MUL(a, b) ((a) * (b))
#define TX_RCP(a) (1.0f / (a))
#define TX_DIV(a, b) ((a) / (b))
#define TX_SQRT(a) std::sqrt(a)
#endif
#ifndef __CUDA_ARCH__
#include <cmath>
#endif

namespace liar_gpu {

// Returns true and writes t when the ray o + t d meets the triangle (v0, v0 + e1, v0 + e2)
// with barycentrics u, v >= 0, u + v <= 1. No range check on t is done here.
TX_HD bool tri_intersect_exact(float ox, float oy, float oz, float dx, float dy, float dz, float v0x, float v0y,
                               float v0z, float e1x, float e1y, float e1z, float e2x, float e2y, float e2z,
                               float& t_out, float& u_out, float& v_out) {
    // p = d x e2
    const float px = TX_SUB(TX_MUL(dy, e2z), TX_MUL(dz, e2y));
    const float py = TX_SUB(TX_MUL(dz, e2x), TX_MUL(dx, e2z));
    const float pz = TX_SUB(TX_MUL(dx, e2y), TX_MUL(dy, e2x));
    const float det = TX_ADD(TX_ADD(TX_MUL(e1x, px), TX_MUL(e1y, py)), TX_MUL(e1z, pz));
    if (det == 0.0f) return false;
    const float inv = TX_RCP(det);
    const float sx = TX_SUB(ox, v0x), sy = TX_SUB(oy, v0y), sz = TX_SUB(oz, v0z);
    const float u = TX_MUL(TX_ADD(TX_ADD(TX_MUL(sx, px), TX_MUL(sy, py)), TX_MUL(sz, pz)), inv);
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    // q = s x e1
    const float qx = TX_SUB(TX_MUL(sy, e1z), TX_MUL(sz, e1y));
    const float qy = TX_SUB(TX_MUL(sz, e1x), TX_MUL(sx, e1z));
    const float qz = TX_SUB(TX_MUL(sx, e1y), TX_MUL(sy, e1x));
    const float v = TX_MUL(TX_ADD(TX_ADD(TX_MUL(dx, qx), TX_MUL(dy, qy)), TX_MUL(dz, qz)), inv);
    if (!(v >= 0.0f && TX_ADD(u, v) <= 1.0f)) return false;
    t_out = TX_MUL(TX_ADD(TX_ADD(TX_MUL(e2x, qx), TX_MUL(e2y, qy)), TX_MUL(e2z, qz)), inv);
    u_out = u;
    v_out = v;
    return true;
}

// The ray o + t d against the sphere |p - c| = r (Sphere::doIntersect, scenery/sphere.cpp:100-128,
// through Lass's intersect(sphere, ray), whose source is not part of the reference): the roots of
// a t^2 + 2 b t + c = 0 with a = d.d, b = (o - c).d, c = |o - c|^2 - r^2, taken in the cancellation-
// free form q = -(b + sign(b) sqrt(b^2 - a c)), t = q / a and c / q (Press et al., Numerical Recipes
// 5.6). Returns the roots in increasing order; false when the ray misses. Correctly rounded
// operations in a fixed order, as in the triangle test.
TX_HD bool sphere_intersect_exact(float ox, float oy, float oz, float dx, float dy, float dz, float cx, float cy,
                                  float cz, float r, float& t0, float& t1) {
    const float sx = TX_SUB(ox, cx), sy = TX_SUB(oy, cy), sz = TX_SUB(oz, cz);
    const float a = TX_ADD(TX_ADD(TX_MUL(dx, dx), TX_MUL(dy, dy)), TX_MUL(dz, dz));
    const float b = TX_ADD(TX_ADD(TX_MUL(sx, dx), TX_MUL(sy, dy)), TX_MUL(sz, dz));
    const float c = TX_SUB(TX_ADD(TX_ADD(TX_MUL(sx, sx), TX_MUL(sy, sy)), TX_MUL(sz, sz)), TX_MUL(r, r));
    const float disc = TX_SUB(TX_MUL(b, b), TX_MUL(a, c));
    if (!(disc >= 0.0f) || !(a > 0.0f)) return false;
    const float root = TX_SQRT(disc);
    const float q = b >= 0.0f ? -TX_ADD(b, root) : TX_SUB(root, b);
    if (q == 0.0f) return false;
    const float ta = TX_DIV(q, a), tb = TX_DIV(c, q);
    t0 = ta < tb ? ta : tb;
    t1 = ta < tb ? tb : ta;
    return true;
}

// BoundedRay::inRange (src/liar/kernel/bounded_ray.h:69-77) with tolerance 1e-6f
// (src/liar/kernel/kernel_common.cpp:32): the open interval, shrunk on both sides.
#define LIAR_TOLERANCE 1e-6f
TX_HD float range_near(float tmin) { return TX_MUL(tmin, TX_ADD(1.0f, LIAR_TOLERANCE)); }
TX_HD float range_far(float tmax) { return TX_MUL(tmax, TX_SUB(1.0f, LIAR_TOLERANCE)); }

}  // namespace liar_gpu
