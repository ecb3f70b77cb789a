// oracle_trace.cpp -- CPU ORACLE (test infrastructure only) for the closest-hit / any-hit path.
//
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm load this
// library, as the checker or the timed CPU baseline; the product never calls it.
//
// What it restates, and from where:
//   * BoundedRay::inRange acceptance, t > near*(1+tol) && t < far*(1-tol), tol = 1e-6f
//     (src/liar/kernel/bounded_ray.h:69-77, src/liar/kernel/kernel_common.cpp:32).
//   * TriangleMesh::doIntersect (src/liar/scenery/triangle_mesh.cpp:291-318): the nearest triangle
//     beyond the near limit, then inRange; the hit index is the position of the triangle in the
//     mesh's triangle array (:309).
//   * TriangleMesh::doIsIntersecting (src/liar/scenery/triangle_mesh.cpp:321-330): occlusion on
//     the open interval (near, far).
//   * The triangle test lives in Lass (lass/prim/triangle_mesh_3d.h, a dependency pinned as
//     lass/1.11.0-250+g078d9309 in conanfile.py:39 and absent from the reference tree). It is
//     restated here as the published two-sided Moller-Trumbore 1997 test, every product and sum
//     rounded to IEEE single in a fixed order, compiled with -ffp-contract=off.
//   * Two traversals: brute force over all triangles (the definition) and a binary tree split at
//     the object median of the widest centroid axis (a different tree from the product's, used
//     only to reach full-size ray sets in seconds).
// Parity status: the hit rule is geometric (nearest t, ties to the lower index), so it does not
// depend on any tree. Agreement with Lass's own arithmetic is unpinned: the reference ships no
// test or golden vector for this path and Lass cannot be built here.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

extern "C" {

struct oracle_ray {
    float ox, oy, oz, tmin, dx, dy, dz, tmax;
};
struct oracle_hit {
    int32_t prim;
    float t;
};

// Moller & Trumbore 1997, two-sided; returns 1 and t/u/v on a hit of the (unbounded) line
int oracle_tri_intersect(const float* o, const float* d, const float* a, const float* b, const float* c, float* t_out,
                         float* u_out, float* v_out) {
    const float e1x = b[0] - a[0], e1y = b[1] - a[1], e1z = b[2] - a[2];
    const float e2x = c[0] - a[0], e2y = c[1] - a[1], e2z = c[2] - a[2];
    const float px = d[1] * e2z - d[2] * e2y;
    const float py = d[2] * e2x - d[0] * e2z;
    const float pz = d[0] * e2y - d[1] * e2x;
    const float det = (e1x * px + e1y * py) + e1z * pz;
    if (det == 0.0f) return 0;
    const float inv = 1.0f / det;
    const float sx = o[0] - a[0], sy = o[1] - a[1], sz = o[2] - a[2];
    const float u = ((sx * px + sy * py) + sz * pz) * inv;
    if (!(u >= 0.0f && u <= 1.0f)) return 0;
    const float qx = sy * e1z - sz * e1y;
    const float qy = sz * e1x - sx * e1z;
    const float qz = sx * e1y - sy * e1x;
    const float v = ((d[0] * qx + d[1] * qy) + d[2] * qz) * inv;
    if (!(v >= 0.0f && u + v <= 1.0f)) return 0;
    *t_out = ((e2x * qx + e2y * qy) + e2z * qz) * inv;
    *u_out = u;
    *v_out = v;
    return 1;
}

// ray / sphere: the roots of a t^2 + 2 b t + c = 0 (a = d.d, b = (o - c).d, c = |o - c|^2 - r^2)
// by q = -(b + sign(b) sqrt(b^2 - a c)), t = q / a, c / q (Numerical Recipes 5.6), in increasing order
int oracle_sphere_intersect(const float* o, const float* d, const float* center, float r, float* t0, float* t1) {
    const float sx = o[0] - center[0], sy = o[1] - center[1], sz = o[2] - center[2];
    const float a = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
    const float b = (sx * d[0] + sy * d[1]) + sz * d[2];
    const float c = ((sx * sx + sy * sy) + sz * sz) - r * r;
    const float disc = b * b - a * c;
    if (!(disc >= 0.0f) || !(a > 0.0f)) return 0;
    const float root = std::sqrt(disc);
    const float q = b >= 0.0f ? -(b + root) : root - b;
    if (q == 0.0f) return 0;
    const float ta = q / a, tb = c / q;
    *t0 = std::min(ta, tb);
    *t1 = std::max(ta, tb);
    return 1;
}

}  // extern "C"

namespace {

const float kTol = 1e-6f;

struct Mesh {
    const float* V;
    const uint32_t* T;
};

inline bool test_tri(const Mesh& m, uint32_t i, const oracle_ray& r, float& t) {
    const float o[3] = {r.ox, r.oy, r.oz}, d[3] = {r.dx, r.dy, r.dz};
    float u, v;
    return oracle_tri_intersect(o, d, m.V + 3 * m.T[3 * i], m.V + 3 * m.T[3 * i + 1], m.V + 3 * m.T[3 * i + 2], &t, &u,
                                &v) != 0;
}

// closest-hit candidate rule shared by both traversals: nearest t beyond tmin, ties to the lower index
inline void offer(int32_t prim, float t, const oracle_ray& r, int32_t& best, float& tbest) {
    if (t > r.tmin && (t < tbest || (t == tbest && prim < best))) {
        tbest = t;
        best = prim;
    }
}

inline oracle_hit finish_closest(int32_t best, float tbest, const oracle_ray& r) {
    // inRange: t > near*(1+tol) && t < far*(1-tol)
    const float lo = r.tmin * (1.0f + kTol), hi = r.tmax * (1.0f - kTol);
    if (best >= 0 && tbest > lo && tbest < hi) return {best, tbest};
    return {-1, INFINITY};
}

template <class F>
void parallel_for(size_t n, int threads, F f) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<size_t> next{0};
    const size_t grain = 256;
    auto work = [&]() {
        while (true) {
            const size_t b = next.fetch_add(grain);
            if (b >= n) break;
            const size_t e = std::min(n, b + grain);
            for (size_t i = b; i < e; ++i) f(i);
        }
    };
    std::vector<std::thread> pool;
    for (int k = 1; k < threads; ++k) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
}

struct BNode {
    float lo[3], hi[3];
    int32_t left, right;  // right < 0: leaf with triangles idx[left .. left + (-right))
};

struct Tree {
    std::vector<BNode> nodes;
    std::vector<uint32_t> idx;
    Mesh mesh;
    std::vector<float> spheres;  // n x 4: centre, radius; primitive index n_tris + k
    uint32_t n_tris = 0;
};

void tri_bounds(const Mesh& m, uint32_t i, float* lo, float* hi) {
    for (int a = 0; a < 3; ++a) {
        const float x0 = m.V[3 * m.T[3 * i] + a], x1 = m.V[3 * m.T[3 * i + 1] + a], x2 = m.V[3 * m.T[3 * i + 2] + a];
        lo[a] = std::min(x0, std::min(x1, x2));
        hi[a] = std::max(x0, std::max(x1, x2));
    }
}

int32_t build_node(Tree& t, std::vector<float>& cent, uint32_t b, uint32_t e, float pad) {
    BNode n;
    for (int a = 0; a < 3; ++a) {
        n.lo[a] = INFINITY;
        n.hi[a] = -INFINITY;
    }
    float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t k = b; k < e; ++k) {
        float lo[3], hi[3];
        tri_bounds(t.mesh, t.idx[k], lo, hi);
        for (int a = 0; a < 3; ++a) {
            n.lo[a] = std::min(n.lo[a], lo[a]);
            n.hi[a] = std::max(n.hi[a], hi[a]);
            clo[a] = std::min(clo[a], cent[3 * t.idx[k] + a]);
            chi[a] = std::max(chi[a], cent[3 * t.idx[k] + a]);
        }
    }
    for (int a = 0; a < 3; ++a) {
        n.lo[a] = std::nextafter(n.lo[a] - pad, -INFINITY);
        n.hi[a] = std::nextafter(n.hi[a] + pad, INFINITY);
    }
    const int32_t me = (int32_t)t.nodes.size();
    t.nodes.push_back(n);
    if (e - b <= 4) {
        t.nodes[me].left = (int32_t)b;
        t.nodes[me].right = -(int32_t)(e - b);
        return me;
    }
    int axis = 0;
    for (int a = 1; a < 3; ++a)
        if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
    const uint32_t mid = b + (e - b) / 2;
    std::nth_element(t.idx.begin() + b, t.idx.begin() + mid, t.idx.begin() + e, [&](uint32_t x, uint32_t y) {
        const float cx = cent[3 * x + axis], cy = cent[3 * y + axis];
        return cx < cy || (cx == cy && x < y);
    });
    const int32_t l = build_node(t, cent, b, mid, pad);
    const int32_t r = build_node(t, cent, mid, e, pad);
    t.nodes[me].left = l;
    t.nodes[me].right = r;
    return me;
}

inline bool box_hit(const BNode& n, const float* o, const float* inv, float tmin, float tmax, float& tnear) {
    float t0 = tmin, t1 = tmax;
    for (int a = 0; a < 3; ++a) {
        float ta = (n.lo[a] - o[a]) * inv[a], tb = (n.hi[a] - o[a]) * inv[a];
        if (ta > tb) std::swap(ta, tb);
        if (!std::isnan(ta)) t0 = std::max(t0, ta);
        if (!std::isnan(tb)) t1 = std::min(t1, tb);
    }
    tnear = t0;
    return t0 <= t1;
}

oracle_hit trace_tree(const Tree& t, const oracle_ray& r, bool any) {
    const float o[3] = {r.ox, r.oy, r.oz};
    float inv[3];
    const float d[3] = {r.dx, r.dy, r.dz};
    for (int a = 0; a < 3; ++a) {
        const float ad = std::fabs(d[a]);
        inv[a] = 1.0f / (ad > 1e-20f ? d[a] : std::copysign(1e-20f, d[a]));
    }
    int32_t best = -1;
    float tbest = any ? r.tmax : r.tmax * (1.0f - kTol);
    // spheres, by brute force: the nearer root beyond tmin, else the farther one
    for (size_t k = 0; 4 * k < t.spheres.size(); ++k) {
        float t0, t1;
        if (!oracle_sphere_intersect(o, d, &t.spheres[4 * k], t.spheres[4 * k + 3], &t0, &t1)) continue;
        const float th = t0 > r.tmin ? t0 : t1;
        const int32_t prim = (int32_t)(t.n_tris + k);
        if (any) {
            if (th > r.tmin && th < r.tmax) return {prim, th};
        } else {
            offer(prim, th, r, best, tbest);
        }
    }
    int32_t stack[128];
    int sp = 0;
    if (!t.nodes.empty()) stack[sp++] = 0;
    while (sp > 0) {
        const BNode& n = t.nodes[stack[--sp]];
        float tn;
        if (!box_hit(n, o, inv, r.tmin, tbest, tn)) continue;
        if (n.right < 0) {
            for (int32_t k = 0; k < -n.right; ++k) {
                const uint32_t prim = t.idx[n.left + k];
                float th;
                if (!test_tri(t.mesh, prim, r, th)) continue;
                if (any) {
                    if (th > r.tmin && th < r.tmax) return {(int32_t)prim, th};
                } else {
                    offer((int32_t)prim, th, r, best, tbest);
                }
            }
        } else if (sp + 2 <= 128) {
            stack[sp++] = n.right;
            stack[sp++] = n.left;
        }
    }
    if (any) return {-1, INFINITY};
    return finish_closest(best, tbest, r);
}

}  // namespace

extern "C" {

// brute force: every ray against every triangle
int oracle_trace_bruteforce(const float* V, uint64_t nv, const uint32_t* T, uint64_t nt, const oracle_ray* rays,
                            uint64_t n, oracle_hit* hits, int any_hit, int threads) {
    (void)nv;
    const Mesh m{V, T};
    parallel_for(n, threads, [&](size_t i) {
        const oracle_ray& r = rays[i];
        int32_t best = -1;
        float tbest = INFINITY;
        for (uint64_t k = 0; k < nt; ++k) {
            float t;
            if (!test_tri(m, (uint32_t)k, r, t)) continue;
            if (any_hit) {
                if (t > r.tmin && t < r.tmax) {
                    best = (int32_t)k;
                    tbest = t;
                    break;
                }
            } else {
                offer((int32_t)k, t, r, best, tbest);
            }
        }
        hits[i] = any_hit ? (best >= 0 ? oracle_hit{best, tbest} : oracle_hit{-1, INFINITY})
                          : finish_closest(best, tbest, r);
    });
    return 0;
}

void* oracle_tree_build(const float* V, uint64_t nv, const uint32_t* T, uint64_t nt) {
    Tree* t = new Tree();
    t->mesh = Mesh{V, T};
    t->idx.resize(nt);
    std::vector<float> cent(3 * nt);
    float mag = 0.0f;
    for (uint64_t i = 0; i < nt; ++i) {
        t->idx[i] = (uint32_t)i;
        float lo[3], hi[3];
        tri_bounds(t->mesh, (uint32_t)i, lo, hi);
        for (int a = 0; a < 3; ++a) {
            cent[3 * i + a] = 0.5f * (lo[a] + hi[a]);
            mag = std::max(mag, std::max(std::fabs(lo[a]), std::fabs(hi[a])));
        }
    }
    (void)nv;
    t->nodes.reserve(nt);
    if (nt) build_node(*t, cent, 0, (uint32_t)nt, mag * 1e-5f);
    return t;
}

// the caller keeps V and T alive while the tree is in use
int oracle_tree_trace(void* tree, const oracle_ray* rays, uint64_t n, oracle_hit* hits, int any_hit, int threads) {
    const Tree& t = *static_cast<Tree*>(tree);
    if (t.nodes.empty()) {
        for (uint64_t i = 0; i < n; ++i) hits[i] = {-1, INFINITY};
        return 0;
    }
    parallel_for(n, threads, [&](size_t i) { hits[i] = trace_tree(t, rays[i], any_hit != 0); });
    return 0;
}

void oracle_tree_free(void* tree) { delete static_cast<Tree*>(tree); }

// analytic spheres (n x 4: centre, radius) beside the tree's n_tris triangles
void oracle_tree_set_spheres(void* tree, const float* spheres, uint64_t n, uint64_t n_tris) {
    Tree& t = *static_cast<Tree*>(tree);
    t.spheres.assign(spheres, spheres + 4 * n);
    t.n_tris = (uint32_t)n_tris;
}

int oracle_hardware_threads(void) { return (int)std::max(1u, std::thread::hardware_concurrency()); }

}  // extern "C"

// closest hit through the oracle tree, for the path-tracer restatement (oracle_render.cpp)
namespace oracle_internal {
struct Ray {
    float ox, oy, oz, tmin, dx, dy, dz, tmax;
};
struct Hit {
    int32_t prim;
    float t;
};
bool tree_any(void* tree, const Ray& r) {
    const Tree& t = *static_cast<Tree*>(tree);
    if (t.nodes.empty() && t.spheres.empty()) return false;
    const oracle_ray rr{r.ox, r.oy, r.oz, r.tmin, r.dx, r.dy, r.dz, r.tmax};
    return trace_tree(t, rr, true).prim >= 0;
}
Hit tree_closest(void* tree, const Ray& r) {
    const Tree& t = *static_cast<Tree*>(tree);
    if (t.nodes.empty() && t.spheres.empty()) return {-1, INFINITY};
    const oracle_ray rr{r.ox, r.oy, r.oz, r.tmin, r.dx, r.dy, r.dz, r.tmax};
    const oracle_hit h = trace_tree(t, rr, false);
    return {h.prim, h.t};
}
}  // namespace oracle_internal
