// linear_octree_gpu.hpp - header-only C++ front end of liboctree_b200.so with
// the reference's names (derivada/octrees-benchmark).
//
// The reference builds and searches like this:
//
//     auto [codes, box] = enc.sortPoints(points, meta);       // point_encoder.hpp:484
//     LinearOctree oct(points, codes, box, enc);              // linear_octree.hpp:614
//     auto idx = oct.neighborsPrune<Kernel_t::sphere>(p, r);  // linear_octree.hpp:1050
//     oct.knn(p, k, indexes, dists);                          // linear_octree.hpp:899
//
// The drop-in is one object that does both steps on the GPU:
//
//     octree_b200::LinearOctree<PointsAoS> oct(points, codes, octree_b200::Encoder::hilbert, 128);
//     auto idx = oct.neighborsPrune<octree_b200::Kernel::sphere>(p, r);
//     oct.knn(p, k, indexes, dists);
//
// As with the reference, `points` is reordered in place along the curve and
// `codes` receives the sorted keys; returned indices index the reordered
// cloud.  The container only needs size(), operator[] returning a point with
// getX()/getY()/getZ(), and set(i, point) - the reference's PointsAoS and
// PointsSoA both qualify.  Batched forms take many centres in one call (that
// is where the GPU pays off).  Errors throw octree_b200::Error.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "octree_b200.h"

namespace octree_b200 {

// Kernel_t (inc/main_options.hpp:97-103) and EncoderType (73-83) values
enum class Kernel : int { circle = OCT_KERNEL_CIRCLE, sphere = OCT_KERNEL_SPHERE, square = OCT_KERNEL_SQUARE,
                          cube = OCT_KERNEL_CUBE };
enum class Encoder : int { morton = OCT_ENC_MORTON_3D, hilbert = OCT_ENC_HILBERT_3D };

class Error : public std::runtime_error {
public:
    Error(int status, const std::string& msg) : std::runtime_error(msg), status_(status) {}
    int status() const { return status_; }

private:
    int status_;
};

// The Box PointEncoder::sortPoints returns (center, radii, min, max).
struct Box {
    double center[3], radii[3], min[3], max[3];
};

// NeighborSet (inc/structures/neighbor_set.hpp:16-90): half-open index ranges.
struct NeighborSet {
    std::vector<std::pair<size_t, size_t>> ranges;
    size_t numberOfPoints = 0;
    size_t size() const { return numberOfPoints; }
    bool empty() const { return numberOfPoints == 0; }
    std::vector<size_t> indices() const {
        std::vector<size_t> out;
        out.reserve(numberOfPoints);
        for (const auto& r : ranges)
            for (size_t i = r.first; i < r.second; ++i) out.push_back(i);
        return out;
    }
};

namespace detail {
inline void check(int st, oct_cloud c, const char* what) {
    if (st == OCT_OK) return;
    std::string msg = std::string(what) + ": " + oct_status_string(st);
    if (c) {
        char buf[512];
        if (oct_last_error(c, buf, sizeof(buf)) == OCT_OK && buf[0]) msg += std::string(" (") + buf + ")";
    }
    throw Error(st, msg);
}
}  // namespace detail

template <class Container>
class LinearOctree {
public:
    // sortPoints + LinearOctree constructor in one step, on `device`.
    LinearOctree(Container& points, std::vector<uint64_t>& codes, Encoder enc = Encoder::hilbert,
                 uint32_t maxPointsLeaf = 128, int device = 0)
        : points_(points) {
        oct_params p{maxPointsLeaf, static_cast<int32_t>(enc), device, 0u};
        detail::check(oct_cloud_create(&p, &cloud_), nullptr, "oct_cloud_create");
        const size_t n = points.size();
        std::vector<double> xyz(3 * n);
        for (size_t i = 0; i < n; ++i) {
            const auto& q = points[i];
            xyz[3 * i] = q.getX();
            xyz[3 * i + 1] = q.getY();
            xyz[3 * i + 2] = q.getZ();
        }
        detail::check(oct_set_points(cloud_, xyz.data(), n, 0), cloud_, "oct_set_points");
        codes.resize(n);
        std::vector<uint32_t> perm(n);
        double b[12];
        detail::check(oct_encode_sort(cloud_, b, codes.data(), perm.data(), nullptr, 0), cloud_, "oct_encode_sort");
        for (int a = 0; a < 3; ++a) {
            box_.center[a] = b[a];
            box_.radii[a] = b[3 + a];
            box_.min[a] = b[6 + a];
            box_.max[a] = b[9 + a];
        }
        // reorder the caller's container in place, moving whole points (ids included)
        std::vector<typename std::decay<decltype(points[0])>::type> tmp;
        tmp.reserve(n);
        for (size_t i = 0; i < n; ++i) tmp.push_back(points[perm[i]]);
        for (size_t i = 0; i < n; ++i) points.set(i, tmp[i]);
        detail::check(oct_build(cloud_, &info_), cloud_, "oct_build");
    }
    LinearOctree(const LinearOctree&) = delete;
    LinearOctree& operator=(const LinearOctree&) = delete;
    ~LinearOctree() {
        if (cloud_) oct_cloud_destroy(cloud_);
    }

    const Box& box() const { return box_; }
    uint32_t nLeaf() const { return info_.n_leaf; }
    uint32_t nInternal() const { return info_.n_internal; }
    uint32_t nTotal() const { return info_.n_total; }
    uint32_t maxDepthSeen() const { return info_.max_depth_seen; }
    oct_cloud handle() const { return cloud_; }

    // ---- single-query forms (the reference's signatures) ----
    template <Kernel K = Kernel::square, class P>
    std::vector<size_t> neighborsPrune(const P& p, double radius) const {
        return one(K, OCT_NEIGHBORS_PRUNE, p, radius);
    }
    template <Kernel K = Kernel::square, class P>
    std::vector<size_t> neighbors(const P& p, double radius) const {
        return one(K, OCT_NEIGHBORS, p, radius);
    }
    template <Kernel K = Kernel::square, class P>
    NeighborSet neighborsStruct(const P& p, double radius) const {
        const double c[3] = {p.getX(), p.getY(), p.getZ()};
        std::vector<NeighborSet> r = structBatch(K, c, 1, radius);
        return std::move(r[0]);
    }
    // neighborsApprox(p, radius, tolerancePercentage, upperBound) (linear_octree.hpp:1089-1093): like
    // the reference, the percentage is used as the precision level, converted to an unsigned integer
    template <Kernel K = Kernel::square, class P>
    NeighborSet neighborsApprox(const P& p, double radius, double tolerancePercentage, bool upperBound) const {
        const double c[3] = {p.getX(), p.getY(), p.getZ()};
        std::vector<NeighborSet> r =
            approxBatch(K, c, 1, radius, static_cast<uint32_t>(tolerancePercentage), upperBound);
        return std::move(r[0]);
    }
    template <class P>
    size_t knn(const P& p, size_t k, std::vector<size_t>& indexes, std::vector<double>& dists) const {
        const double c[3] = {p.getX(), p.getY(), p.getZ()};
        std::vector<uint32_t> idx(k);
        std::vector<double> d2(k);
        uint32_t cnt = 0;
        detail::check(oct_knn(cloud_, c, 1, static_cast<uint32_t>(k), idx.data(), d2.data(), &cnt, 0), cloud_,
                      "oct_knn");
        if (indexes.size() < k) indexes.resize(k);
        if (dists.size() < k) dists.resize(k);
        for (uint32_t j = 0; j < cnt; ++j) {
            indexes[j] = idx[j];
            dists[j] = d2[j];
        }
        return cnt;
    }

    // ---- batched forms: centres xyz (nq x 3), CSR result ----
    void radiusBatch(Kernel k, int algo, const double* centers, size_t nq, double radius,
                     std::vector<uint64_t>& offsets, std::vector<uint32_t>& idx) const {
        offsets.assign(nq + 1, 0);
        uint64_t total = 0;
        int st = oct_radius_search(cloud_, static_cast<int>(k), algo, centers, nq, nullptr, radius, offsets.data(),
                                   nullptr, 0, &total, 0);
        if (st != OCT_OK && st != OCT_ERR_CAPACITY) detail::check(st, cloud_, "oct_radius_search");
        idx.assign(total, 0);
        if (total)
            detail::check(oct_radius_search(cloud_, static_cast<int>(k), algo, centers, nq, nullptr, radius,
                                            offsets.data(), idx.data(), total, &total, 0),
                          cloud_, "oct_radius_search");
    }
    std::vector<NeighborSet> structBatch(Kernel k, const double* centers, size_t nq, double radius) const {
        return rangesBatch(k, centers, nq, radius, false, 0, false);
    }
    // neighborsApprox over nq centres at one precision level
    std::vector<NeighborSet> approxBatch(Kernel k, const double* centers, size_t nq, double radius,
                                         uint32_t precisionLevel, bool upperBound) const {
        return rangesBatch(k, centers, nq, radius, true, precisionLevel, upperBound);
    }

private:
    std::vector<NeighborSet> rangesBatch(Kernel k, const double* centers, size_t nq, double radius, bool approx,
                                         uint32_t level, bool upper) const {
        std::vector<uint64_t> offs(nq + 1), npts(nq);
        uint64_t total = 0;
        auto call = [&](uint32_t* pairs, uint64_t cap) {
            return approx ? oct_approx_search(cloud_, static_cast<int>(k), centers, nq, nullptr, radius, level,
                                              upper ? 1 : 0, offs.data(), pairs, cap, &total, npts.data(), 0)
                          : oct_struct_search(cloud_, static_cast<int>(k), centers, nq, nullptr, radius, offs.data(),
                                              pairs, cap, &total, npts.data(), 0);
        };
        const char* what = approx ? "oct_approx_search" : "oct_struct_search";
        int st = call(nullptr, 0);
        if (st != OCT_OK && st != OCT_ERR_CAPACITY) detail::check(st, cloud_, what);
        std::vector<uint32_t> pairs(2 * total);
        if (total) detail::check(call(pairs.data(), total), cloud_, what);
        std::vector<NeighborSet> out(nq);
        for (size_t q = 0; q < nq; ++q) {
            for (uint64_t j = offs[q]; j < offs[q + 1]; ++j) out[q].ranges.emplace_back(pairs[2 * j], pairs[2 * j + 1]);
            out[q].numberOfPoints = npts[q];
        }
        return out;
    }

public:
    void knnBatch(const double* centers, size_t nq, uint32_t k, std::vector<uint32_t>& idx, std::vector<double>& d2,
                  std::vector<uint32_t>& counts) const {
        idx.resize(nq * k);
        d2.resize(nq * k);
        counts.resize(nq);
        detail::check(oct_knn(cloud_, centers, nq, k, idx.data(), d2.data(), counts.data(), 0), cloud_, "oct_knn");
    }

private:
    template <class P>
    std::vector<size_t> one(Kernel k, int algo, const P& p, double radius) const {
        const double c[3] = {p.getX(), p.getY(), p.getZ()};
        std::vector<uint64_t> offs;
        std::vector<uint32_t> idx;
        radiusBatch(k, algo, c, 1, radius, offs, idx);
        return std::vector<size_t>(idx.begin(), idx.end());
    }

    Container& points_;
    oct_cloud cloud_ = nullptr;
    oct_tree_info info_{};
    Box box_{};
};

}  // namespace octree_b200
