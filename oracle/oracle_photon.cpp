// oracle_photon.cpp -- CPU ORACLE (test infrastructure only) of the photon-map gather.
//
// Restates KdTree::rangeSearch(point, maxRadius, maxCount) as the reference's PhotonMapper uses it
// (src/liar/tracers/photon_mapper.cpp:1257, 1312, 1352; the tree is Lass's spat::KdTree, pinned
// as lass/1.11.0-250+g078d9309 and absent from the reference tree): the at most k photons with
// squared distance < r_max^2 nearest to the query. Exact brute force over all photons, squared
// distances evaluated as ((dx*dx + dy*dy) + dz*dz) in IEEE single (compiled without
// contraction), ordered by (distance, index). Neighbour sets are therefore exact; agreement
// with Lass's own tie handling at equal distance is unpinned.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <thread>
#include <utility>
#include <vector>

extern "C" int oracle_knn(const float* photons, uint64_t n, const float* queries, uint64_t nq, int k, float r_max,
                          int32_t* idx, float* d2, int32_t* count, int threads) {
    const float r2 = r_max * r_max;
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<uint64_t> next{0};
    auto work = [&]() {
        std::vector<std::pair<float, int32_t>> cand;
        while (true) {
            const uint64_t q = next.fetch_add(1);
            if (q >= nq) break;
            const float qx = queries[3 * q], qy = queries[3 * q + 1], qz = queries[3 * q + 2];
            cand.clear();
            for (uint64_t i = 0; i < n; ++i) {
                const float dx = photons[3 * i] - qx, dy = photons[3 * i + 1] - qy, dz = photons[3 * i + 2] - qz;
                const float dd = (dx * dx + dy * dy) + dz * dz;
                if (dd < r2) cand.emplace_back(dd, (int32_t)i);
            }
            const size_t m = std::min<size_t>(cand.size(), (size_t)k);
            std::partial_sort(cand.begin(), cand.begin() + m, cand.end());
            for (int j = 0; j < k; ++j) {
                idx[q * k + j] = (size_t)j < m ? cand[j].second : -1;
                d2[q * k + j] = (size_t)j < m ? cand[j].first : INFINITY;
            }
            if (count) count[q] = (int32_t)m;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return 0;
}

// The same search over a uniform grid of cells of size r_max (sorted cell keys + binary search):
// the CPU baseline at sizes where brute force is out of reach. Same keys, same results.
extern "C" int oracle_knn_grid(const float* photons, uint64_t n, const float* queries, uint64_t nq, int k, float r_max,
                               int32_t* idx, float* d2, int32_t* count, int threads) {
    const float r2 = r_max * r_max;
    const double inv = 1.0 / ((double)r_max * 1.001);
    auto cell = [&](const float* p, int64_t c[3]) {
        for (int a = 0; a < 3; ++a) c[a] = (int64_t)std::floor((double)p[a] * inv);
    };
    auto key = [](int64_t x, int64_t y, int64_t z) {
        return ((uint64_t)(x + (1 << 20)) << 42) | ((uint64_t)(y + (1 << 20)) << 21) | (uint64_t)(z + (1 << 20));
    };
    std::vector<std::pair<uint64_t, uint32_t>> sorted(n);
    for (uint64_t i = 0; i < n; ++i) {
        int64_t c[3];
        cell(photons + 3 * i, c);
        sorted[i] = {key(c[0], c[1], c[2]), (uint32_t)i};
    }
    std::sort(sorted.begin(), sorted.end());
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<uint64_t> next{0};
    auto work = [&]() {
        std::vector<std::pair<float, int32_t>> cand;
        while (true) {
            const uint64_t q = next.fetch_add(1);
            if (q >= nq) break;
            const float* qp = queries + 3 * q;
            int64_t c[3];
            cell(qp, c);
            cand.clear();
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const uint64_t kk = key(c[0] + dx, c[1] + dy, c[2] + dz);
                        auto it = std::lower_bound(sorted.begin(), sorted.end(), std::make_pair(kk, 0u));
                        for (; it != sorted.end() && it->first == kk; ++it) {
                            const float* p = photons + 3 * (uint64_t)it->second;
                            const float ex = p[0] - qp[0], ey = p[1] - qp[1], ez = p[2] - qp[2];
                            const float dd = (ex * ex + ey * ey) + ez * ez;
                            if (dd < r2) cand.emplace_back(dd, (int32_t)it->second);
                        }
                    }
            const size_t m = std::min<size_t>(cand.size(), (size_t)k);
            std::partial_sort(cand.begin(), cand.begin() + m, cand.end());
            for (int j = 0; j < k; ++j) {
                idx[q * k + j] = (size_t)j < m ? cand[j].second : -1;
                d2[q * k + j] = (size_t)j < m ? cand[j].first : INFINITY;
            }
            if (count) count[q] = (int32_t)m;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return 0;
}
