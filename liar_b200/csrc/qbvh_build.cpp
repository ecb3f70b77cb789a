// qbvh_build.cpp -- host builder of the 4-wide SAH tree consumed by the traversal kernels.
//
// Replaces the Lass QbvhTree<..., SAHSplitHeuristics>::reset that TriangleMesh runs on
// construction (src/liar/scenery/triangle_mesh.cpp:69-85) and ObjectTree::doPreProcess runs
// on the object level (src/liar/scenery/object_trees.h:100-108). Lass's source is not in the
// reference, so this follows the published method instead:
//   1. a binary tree by binned SAH (Wald 2007, "On fast construction of SAH-based bounding
//      volume hierarchies"), leaves of at most max_leaf_size triangles;
//   2. collapse to 4 children per node by repeatedly opening the child of largest surface
//      area (Dammertz, Hanika, Keller 2008 "Shallow bounding volume hierarchies for fast SIMD
//      ray tracing of incoherent rays"; Wald, Benthin, Boulos 2008 "Getting rid of packets").
// Subtrees above 64k triangles are built on separate std::threads.
#include "qbvh.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

#include "../../include/liar_gpu.h"

namespace liar_gpu {
namespace {

struct Box {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const float* l, const float* h) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], l[a]);
            hi[a] = std::max(hi[a], h[a]);
        }
    }
    void grow(const Box& b) { grow(b.lo, b.hi); }
    void grow_point(const float* p) { grow(p, p); }
    bool empty() const { return lo[0] > hi[0]; }
    double area() const {
        if (empty()) return 0.0;
        const double dx = (double)hi[0] - lo[0], dy = (double)hi[1] - lo[1], dz = (double)hi[2] - lo[2];
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
};

struct PrimRef {
    float lo[3], hi[3], c[3];
};

struct BNode {
    Box box;
    int32_t left = -1, right = -1;   // children (inner) or -1 (leaf)
    uint32_t first = 0, count = 0;   // leaf range in the index array
};

struct Builder {
    const std::vector<PrimRef>& prims;
    std::vector<uint32_t>& idx;
    std::vector<BNode>& nodes;
    std::atomic<int64_t> next_node{0};
    std::atomic<int> live_threads{1};
    int max_threads;
    int max_leaf;
    int bins;
    double c_trav;

    Builder(const std::vector<PrimRef>& p, std::vector<uint32_t>& i, std::vector<BNode>& n, int threads, int leaf,
            int nbins, double ct)
        : prims(p), idx(i), nodes(n), max_threads(threads), max_leaf(leaf), bins(nbins), c_trav(ct) {}

    int32_t alloc() { return (int32_t)next_node.fetch_add(1); }

    void make_leaf(int32_t ni, uint32_t begin, uint32_t end) {
        nodes[ni].left = nodes[ni].right = -1;
        nodes[ni].first = begin;
        nodes[ni].count = end - begin;
    }

    // builds node ni over idx[begin, end)
    void build(int32_t ni, uint32_t begin, uint32_t end, int depth) {
        Box nb, cb;
        for (uint32_t k = begin; k < end; ++k) {
            const PrimRef& p = prims[idx[k]];
            nb.grow(p.lo, p.hi);
            cb.grow_point(p.c);
        }
        nodes[ni].box = nb;
        const uint32_t n = end - begin;
        if (n == 1) {
            make_leaf(ni, begin, end);
            return;
        }
        // best binned split over the three axes
        int best_axis = -1, best_bin = -1;
        double best_cost = INFINITY;
        const int K = bins;
        std::vector<Box> bbox(K);
        std::vector<uint32_t> bcnt(K);
        std::vector<double> right_area(K);
        std::vector<uint32_t> right_cnt(K);
        for (int a = 0; a < 3; ++a) {
            const float ext = cb.hi[a] - cb.lo[a];
            if (!(ext > 0.0f)) continue;
            const double scale = (double)K / (double)ext * (1.0 - 1e-6);
            std::fill(bbox.begin(), bbox.end(), Box());
            std::fill(bcnt.begin(), bcnt.end(), 0u);
            for (uint32_t k = begin; k < end; ++k) {
                const PrimRef& p = prims[idx[k]];
                int b = (int)(((double)p.c[a] - cb.lo[a]) * scale);
                b = std::min(std::max(b, 0), K - 1);
                bbox[b].grow(p.lo, p.hi);
                bcnt[b]++;
            }
            Box acc;
            uint32_t cnt = 0;
            for (int b = K - 1; b > 0; --b) {
                acc.grow(bbox[b]);
                cnt += bcnt[b];
                right_area[b] = acc.area();
                right_cnt[b] = cnt;
            }
            acc = Box();
            cnt = 0;
            for (int b = 0; b < K - 1; ++b) {
                acc.grow(bbox[b]);
                cnt += bcnt[b];
                const uint32_t rc = right_cnt[b + 1];
                if (cnt == 0 || rc == 0) continue;
                const double cost = acc.area() * cnt + right_area[b + 1] * rc;
                if (cost < best_cost) {
                    best_cost = cost;
                    best_axis = a;
                    best_bin = b;
                }
            }
        }
        const double parent_area = nb.area();
        const double split_cost = parent_area > 0 ? c_trav + best_cost / parent_area : INFINITY;
        const double leaf_cost = (double)n;
        uint32_t mid;
        if (best_axis < 0) {
            // all centroids coincide: split by position in the array
            if (n <= (uint32_t)max_leaf) {
                make_leaf(ni, begin, end);
                return;
            }
            mid = begin + n / 2;
        } else {
            if (n <= (uint32_t)max_leaf && leaf_cost <= split_cost) {
                make_leaf(ni, begin, end);
                return;
            }
            const int a = best_axis;
            const double scale = (double)K / (double)(cb.hi[a] - cb.lo[a]) * (1.0 - 1e-6);
            auto it = std::partition(idx.begin() + begin, idx.begin() + end, [&](uint32_t i) {
                int b = (int)(((double)prims[i].c[a] - cb.lo[a]) * scale);
                b = std::min(std::max(b, 0), K - 1);
                return b <= best_bin;
            });
            mid = (uint32_t)(it - idx.begin());
            if (mid == begin || mid == end) mid = begin + n / 2;
        }
        const int32_t l = alloc(), r = alloc();
        nodes[ni].left = l;
        nodes[ni].right = r;
        nodes[ni].count = 0;
        if (n > 65536 && live_threads.load() < max_threads) {
            live_threads.fetch_add(1);
            std::thread t([this, l, begin, mid, depth]() { build(l, begin, mid, depth + 1); });
            build(r, mid, end, depth + 1);
            t.join();
            live_threads.fetch_sub(1);
        } else {
            build(l, begin, mid, depth + 1);
            build(r, mid, end, depth + 1);
        }
    }
};

struct Collapser {
    const std::vector<BNode>& bnodes;
    std::vector<QNode> qnodes;
    float pad;
    double root_area;
    double sah = 0.0;
    uint64_t leaves = 0;
    uint32_t max_depth = 0;
    uint32_t max_stack = 0;
    double c_trav;

    Collapser(const std::vector<BNode>& b, float p, double ra, double ct) : bnodes(b), pad(p), root_area(ra), c_trav(ct) {}

    static float down(float x) { return std::nextafter(x, -INFINITY); }
    static float up(float x) { return std::nextafter(x, INFINITY); }

    // returns the index of the new QNode
    int32_t emit(int32_t bi, uint32_t depth, uint32_t stack_so_far) {
        std::vector<int32_t> kids;
        const BNode& b = bnodes[bi];
        if (b.left < 0) {
            kids.push_back(bi);  // a root that is a single leaf
        } else {
            kids.push_back(b.left);
            kids.push_back(b.right);
        }
        while (kids.size() < 4) {
            int pick = -1;
            double pick_area = -1.0;
            for (size_t k = 0; k < kids.size(); ++k) {
                const BNode& c = bnodes[kids[k]];
                if (c.left >= 0 && c.box.area() > pick_area) {
                    pick_area = c.box.area();
                    pick = (int)k;
                }
            }
            if (pick < 0) break;
            const BNode& c = bnodes[kids[pick]];
            kids[pick] = c.left;
            kids.push_back(c.right);
        }
        const int32_t qi = (int32_t)qnodes.size();
        qnodes.emplace_back();
        sah += c_trav * bnodes[bi].box.area() / root_area;
        max_depth = std::max(max_depth, depth + 1);
        const uint32_t stack_here = stack_so_far + (uint32_t)(kids.size() - 1);
        max_stack = std::max(max_stack, stack_here);
        float lo[3][4], hi[3][4];
        int32_t child[4], count[4];
        for (int c = 0; c < 4; ++c) {
            for (int a = 0; a < 3; ++a) {
                lo[a][c] = INFINITY;
                hi[a][c] = -INFINITY;
            }
            child[c] = (int32_t)0x80000000u;  // empty leaf slot: zero triangles
            count[c] = 0;
        }
        for (size_t k = 0; k < kids.size(); ++k) {
            const BNode& c = bnodes[kids[k]];
            for (int a = 0; a < 3; ++a) {
                lo[a][k] = down(c.box.lo[a] - pad);
                hi[a][k] = up(c.box.hi[a] + pad);
            }
            if (c.left < 0) {
                child[k] = (int32_t)(0x80000000u | (c.count << 27) | c.first);
                count[k] = (int32_t)c.count;
                sah += (double)c.count * c.box.area() / root_area;
                ++leaves;
            }
        }
        for (size_t k = 0; k < kids.size(); ++k) {
            const BNode& c = bnodes[kids[k]];
            if (c.left >= 0) child[k] = emit(kids[k], depth + 1, stack_here);
        }
        QNode& q = qnodes[qi];
        q.lo_x = {lo[0][0], lo[0][1], lo[0][2], lo[0][3]};
        q.hi_x = {hi[0][0], hi[0][1], hi[0][2], hi[0][3]};
        q.lo_y = {lo[1][0], lo[1][1], lo[1][2], lo[1][3]};
        q.hi_y = {hi[1][0], hi[1][1], hi[1][2], hi[1][3]};
        q.lo_z = {lo[2][0], lo[2][1], lo[2][2], lo[2][3]};
        q.hi_z = {hi[2][0], hi[2][1], hi[2][2], hi[2][3]};
        q.child = {child[0], child[1], child[2], child[3]};
        q.count = {count[0], count[1], count[2], count[3]};
        return qi;
    }
};

}  // namespace

int build_qbvh(const float* V, uint64_t nv, const uint32_t* T, uint64_t nt, const BuildOptions& opts, QBVHHost& out,
               char* msg, size_t msg_len) {
    return build_qbvh(V, nv, T, nt, nullptr, 0, opts, out, msg, msg_len);
}

int build_qbvh(const float* V, uint64_t nv, const uint32_t* T, uint64_t nt, const float* S, uint64_t ns,
               const BuildOptions& opts, QBVHHost& out, char* msg, size_t msg_len) {
    auto fail = [&](int code, const char* what) {
        if (msg && msg_len) std::snprintf(msg, msg_len, "%s", what);
        return code;
    };
    if (nt + ns == 0) return fail(LIAR_ERR_INVALID, "mesh has no triangles");
    if (nt + ns >= (1ull << 27)) return fail(LIAR_ERR_INVALID, "too many primitives (limit 2^27 - 1 per mesh)");
    if (nt > 0 && (!V || !T)) return fail(LIAR_ERR_INVALID, "null vertex or triangle array");
    if (ns > 0 && !S) return fail(LIAR_ERR_INVALID, "null sphere array");
    for (uint64_t k = 0; k < ns; ++k)
        if (!std::isfinite(S[4 * k]) || !std::isfinite(S[4 * k + 1]) || !std::isfinite(S[4 * k + 2]) ||
            !(S[4 * k + 3] > 0.0f) || !std::isfinite(S[4 * k + 3]))
            return fail(LIAR_ERR_INVALID, "sphere centre not finite or radius not positive");
    const uint64_t np = nt + ns;
    const int max_leaf = opts.max_leaf_size <= 0 ? 4 : opts.max_leaf_size;
    if (max_leaf > 8) return fail(LIAR_ERR_INVALID, "max_leaf_size must be 1..8");
    const int bins = opts.sah_bins <= 0 ? 32 : std::min(opts.sah_bins, 256);
    int threads = opts.threads > 0 ? opts.threads : (int)std::thread::hardware_concurrency();
    if (threads <= 0) threads = 1;
    for (uint64_t k = 0; k < nv * 3; ++k)
        if (!std::isfinite(V[k])) return fail(LIAR_ERR_INVALID, "vertex coordinate is not finite");
    for (uint64_t k = 0; k < nt * 3; ++k)
        if (T[k] >= nv) return fail(LIAR_ERR_INVALID, "triangle vertex index out of range");

    std::vector<PrimRef> prims(np);
    Box root;
    for (uint64_t i = 0; i < nt; ++i) {
        PrimRef& p = prims[i];
        for (int a = 0; a < 3; ++a) {
            const float x0 = V[3 * T[3 * i + 0] + a], x1 = V[3 * T[3 * i + 1] + a], x2 = V[3 * T[3 * i + 2] + a];
            p.lo[a] = std::min(x0, std::min(x1, x2));
            p.hi[a] = std::max(x0, std::max(x1, x2));
            p.c[a] = 0.5f * (p.lo[a] + p.hi[a]);
        }
        root.grow(p.lo, p.hi);
    }
    for (uint64_t k = 0; k < ns; ++k) {
        // a sphere's box, rounded outward by the relative error of centre +- radius
        PrimRef& p = prims[nt + k];
        const float r = S[4 * k + 3];
        for (int a = 0; a < 3; ++a) {
            const float c = S[4 * k + a];
            const float slack = (std::fabs(c) + r) * 2.4e-7f;
            p.lo[a] = (c - r) - slack;
            p.hi[a] = (c + r) + slack;
            p.c[a] = c;
        }
        root.grow(p.lo, p.hi);
    }
    std::vector<uint32_t> idx(np);
    for (uint64_t i = 0; i < np; ++i) idx[i] = (uint32_t)i;
    std::vector<BNode> bnodes(2 * np);
    Builder b(prims, idx, bnodes, threads, max_leaf, bins, opts.traversal_cost > 0 ? opts.traversal_cost : 1.0);
    const int32_t r = b.alloc();
    b.build(r, 0, (uint32_t)np, 0);
    bnodes.resize((size_t)b.next_node.load());

    // conservative padding of every child box (absolute, relative to the scene's magnitude)
    float mag = 0.0f;
    for (int a = 0; a < 3; ++a) {
        mag = std::max(mag, root.hi[a] - root.lo[a]);
        mag = std::max(mag, std::fabs(root.lo[a]));
        mag = std::max(mag, std::fabs(root.hi[a]));
    }
    const float pad = mag * 7.62939453125e-06f;  // 2^-17
    const double ra = root.area() > 0 ? root.area() : 1.0;
    Collapser col(bnodes, pad, ra, opts.traversal_cost > 0 ? opts.traversal_cost : 1.0);
    col.qnodes.reserve(bnodes.size() / 3 + 1);
    col.emit(r, 0, 0);

    out.n_nodes = col.qnodes.size();
    out.nodes = (QNode*)std::aligned_alloc(128, out.n_nodes * sizeof(QNode));
    if (!out.nodes) return fail(LIAR_ERR_OOM, "host allocation of nodes failed");
    std::memcpy(out.nodes, col.qnodes.data(), out.n_nodes * sizeof(QNode));
    out.n_tris = np;
    out.tris = (QTri*)std::aligned_alloc(128, ((np * sizeof(QTri) + 127) / 128) * 128);
    if (!out.tris) {
        std::free(out.nodes);
        out.nodes = nullptr;
        return fail(LIAR_ERR_OOM, "host allocation of triangles failed");
    }
    for (uint64_t k = 0; k < np; ++k) {
        const uint32_t i = idx[k];
        QTri& q = out.tris[k];
        int32_t ii = (int32_t)i;
        float wbits;
        std::memcpy(&wbits, &ii, 4);
        if (i >= nt) {
            // a sphere: centre and index bits, then the radius with the sphere flag in e1.w
            const float* sp = S + 4 * (i - nt);
            q.v0 = {sp[0], sp[1], sp[2], wbits};
            q.e1 = {sp[3], 0.0f, 0.0f, 1.0f};
            q.e2 = {0.0f, 0.0f, 0.0f, 0.0f};
            continue;
        }
        const float* a = V + 3 * T[3 * i + 0];
        const float* bb = V + 3 * T[3 * i + 1];
        const float* c = V + 3 * T[3 * i + 2];
        q.v0 = {a[0], a[1], a[2], wbits};
        q.e1 = {bb[0] - a[0], bb[1] - a[1], bb[2] - a[2], 0.0f};
        q.e2 = {c[0] - a[0], c[1] - a[1], c[2] - a[2], 0.0f};
    }
    out.n_leaves = col.leaves;
    out.max_depth = col.max_depth;
    out.stack_needed = col.max_stack;
    out.sah_cost = col.sah;
    return LIAR_OK;
}

void free_qbvh(QBVHHost& q) {
    std::free(q.nodes);
    std::free(q.tris);
    q.nodes = nullptr;
    q.tris = nullptr;
    q.n_nodes = q.n_tris = 0;
}

}  // namespace liar_gpu
