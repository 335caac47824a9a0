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
// The same four calls compile against this header in namespace octree_b200
// (PointEncoding::getEncoder / MortonEncoder3D / HilbertEncoder3D, Kernel_t,
// mainOptions.maxPointsLeaf), with sortPoints and the octree on the GPU:
//
//     using namespace octree_b200;
//     auto& enc = PointEncoding::getEncoder(EncoderType::HILBERT_ENCODER_3D);
//     auto [codes, box] = enc.sortPoints(points, meta);
//     LinearOctree oct(points, codes, box, enc);
//     auto idx = oct.neighborsPrune<Kernel_t::sphere>(p, r);
//     oct.knn(p, k, indexes, dists);
//
// or as one object that does both steps:
//
//     octree_b200::LinearOctree<PointsAoS> oct(points, codes, octree_b200::Encoder::hilbert, 128);
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
#include <optional>
#include <stdexcept>
#include <type_traits>
#include <string>
#include <utility>
#include <vector>

#include "octree_b200.h"

namespace octree_b200 {

// Kernel_t (inc/main_options.hpp:97-103) and EncoderType (73-83) values
enum class Kernel : int { circle = OCT_KERNEL_CIRCLE, sphere = OCT_KERNEL_SPHERE, square = OCT_KERNEL_SQUARE,
                          cube = OCT_KERNEL_CUBE };
enum class Encoder : int { morton = OCT_ENC_MORTON_3D, hilbert = OCT_ENC_HILBERT_3D };
using Kernel_t = Kernel;
// EncoderType (inc/main_options.hpp:73-83): the 3D encoders the octree takes
enum EncoderType : int { MORTON_ENCODER_3D = OCT_ENC_MORTON_3D, HILBERT_ENCODER_3D = OCT_ENC_HILBERT_3D };

// The reference's global configuration the octree reads (mainOptions.maxPointsLeaf,
// inc/main_options.hpp), plus the CUDA device the octrees of this front end use.
struct MainOptions {
    uint32_t maxPointsLeaf = 128;
    int device = 0;
};
inline MainOptions mainOptions;

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

// Reorder `c` in place so that c[i] becomes the old c[perm[i]] (whole elements move).
template <class C>
void permute_points(C& c, const std::vector<uint32_t>& perm) {
    std::vector<typename std::decay<decltype(c[0])>::type> tmp;
    tmp.reserve(perm.size());
    for (size_t i = 0; i < perm.size(); ++i) tmp.push_back(c[perm[i]]);
    for (size_t i = 0; i < perm.size(); ++i) c.set(i, tmp[i]);
}

template <class Container>
std::vector<double> xyz_of(const Container& points) {
    const size_t n = points.size();
    std::vector<double> xyz(3 * n);
    for (size_t i = 0; i < n; ++i) {
        const auto& q = points[i];
        xyz[3 * i] = q.getX();
        xyz[3 * i + 1] = q.getY();
        xyz[3 * i + 2] = q.getZ();
    }
    return xyz;
}

inline Box box_of(const double* b) {
    Box box{};
    for (int a = 0; a < 3; ++a) {
        box.center[a] = b[a];
        box.radii[a] = b[3 + a];
        box.min[a] = b[6 + a];
        box.max[a] = b[9 + a];
    }
    return box;
}
}  // namespace detail

// PointEncoder (inc/encoding/point_encoder.hpp): sortPoints encodes, sorts and
// reorders on the GPU.
class PointEncoder {
public:
    explicit PointEncoder(EncoderType t) : type_(t) {}
    EncoderType type() const { return type_; }

    // sortPoints(points, meta) (point_encoder.hpp:484-503): the Box of the cloud and the sorted codes; the
    // container (and the metadata, when present) are reordered in place along the curve.
    template <class Container, class Meta>
    std::pair<std::vector<uint64_t>, Box> sortPoints(Container& points, std::optional<std::vector<Meta>>& meta) const {
        std::vector<uint32_t> perm;
        auto out = sort(points, perm);
        if (meta && !meta->empty()) {
            std::vector<Meta> tmp;
            tmp.reserve(perm.size());
            for (uint32_t j : perm) tmp.push_back((*meta)[j]);
            *meta = std::move(tmp);
        }
        return out;
    }
    template <class Container>
    std::pair<std::vector<uint64_t>, Box> sortPoints(Container& points) const {
        std::vector<uint32_t> perm;
        return sort(points, perm);
    }

private:
    template <class Container>
    std::pair<std::vector<uint64_t>, Box> sort(Container& points, std::vector<uint32_t>& perm) const {
        oct_params p{mainOptions.maxPointsLeaf, static_cast<int32_t>(type_), mainOptions.device, 0u};
        oct_cloud c = nullptr;
        detail::check(oct_cloud_create(&p, &c), nullptr, "oct_cloud_create");
        struct Guard {
            oct_cloud c;
            ~Guard() { oct_cloud_destroy(c); }
        } guard{c};
        const size_t n = points.size();
        std::vector<double> xyz = detail::xyz_of(points);
        detail::check(oct_set_points(c, xyz.data(), n, 0), c, "oct_set_points");
        std::vector<uint64_t> codes(n);
        perm.assign(n, 0);
        double b[12];
        detail::check(oct_encode_sort(c, b, codes.data(), perm.data(), nullptr, 0), c, "oct_encode_sort");
        detail::permute_points(points, perm);
        return {std::move(codes), detail::box_of(b)};
    }

    EncoderType type_;
};

namespace PointEncoding {
struct MortonEncoder3D : PointEncoder {
    MortonEncoder3D() : PointEncoder(MORTON_ENCODER_3D) {}
};
struct HilbertEncoder3D : PointEncoder {
    HilbertEncoder3D() : PointEncoder(HILBERT_ENCODER_3D) {}
};
// getEncoder (inc/encoding/point_encoder_factory.hpp:12): one instance per type
inline PointEncoder& getEncoder(EncoderType t) {
    static MortonEncoder3D morton;
    static HilbertEncoder3D hilbert;
    if (t == MORTON_ENCODER_3D) return morton;
    if (t == HILBERT_ENCODER_3D) return hilbert;
    throw Error(OCT_ERR_INVALID_ARG, "the octree takes the 3D Morton or Hilbert encoder");
}
}  // namespace PointEncoding

template <class Container>
class LinearOctree {
public:
    // LinearOctree(points, codes, box, enc) (linear_octree.hpp:614-623): the points already sorted by
    // sortPoints, their codes and Box; mainOptions.maxPointsLeaf points per leaf, on mainOptions.device.
    LinearOctree(Container& points, std::vector<uint64_t>& codes, Box box, PointEncoder& enc) : points_(points) {
        oct_params p{mainOptions.maxPointsLeaf, static_cast<int32_t>(enc.type()), mainOptions.device, 0u};
        detail::check(oct_cloud_create(&p, &cloud_), nullptr, "oct_cloud_create");
        const size_t n = points.size();
        if (codes.size() != n) {
            oct_cloud_destroy(cloud_);
            cloud_ = nullptr;
            throw Error(OCT_ERR_INVALID_ARG, "codes and points differ in size");
        }
        std::vector<double> xyz = detail::xyz_of(points);
        double b[12];
        for (int a = 0; a < 3; ++a) {
            b[a] = box.center[a];
            b[3 + a] = box.radii[a];
            b[6 + a] = box.min[a];
            b[9 + a] = box.max[a];
        }
        box_ = box;
        try {
            detail::check(oct_set_sorted_points(cloud_, xyz.data(), codes.data(), n, b, 0), cloud_,
                          "oct_set_sorted_points");
            detail::check(oct_build(cloud_, &info_), cloud_, "oct_build");
        } catch (...) {
            oct_cloud_destroy(cloud_);
            cloud_ = nullptr;
            throw;
        }
    }

    // sortPoints + LinearOctree constructor in one step, on `device`.
    LinearOctree(Container& points, std::vector<uint64_t>& codes, Encoder enc = Encoder::hilbert,
                 uint32_t maxPointsLeaf = 128, int device = 0)
        : points_(points) {
        oct_params p{maxPointsLeaf, static_cast<int32_t>(enc), device, 0u};
        detail::check(oct_cloud_create(&p, &cloud_), nullptr, "oct_cloud_create");
        const size_t n = points.size();
        std::vector<double> xyz = detail::xyz_of(points);
        detail::check(oct_set_points(cloud_, xyz.data(), n, 0), cloud_, "oct_set_points");
        codes.resize(n);
        std::vector<uint32_t> perm(n);
        double b[12];
        detail::check(oct_encode_sort(cloud_, b, codes.data(), perm.data(), nullptr, 0), cloud_, "oct_encode_sort");
        box_ = detail::box_of(b);
        // reorder the caller's container in place, moving whole points (ids included)
        detail::permute_points(points, perm);
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
    // Vector-radii overloads (linear_octree.hpp:1044-1048, 1056-1060, 1069-1074): square and cube kernels,
    // per-axis radii (any type with getX/getY/getZ)
    template <Kernel K = Kernel::cube, class P, class V, class = std::enable_if_t<!std::is_arithmetic<V>::value>>
    std::vector<size_t> neighborsPrune(const P& p, const V& radii) const {
        return oneAxes(K, OCT_NEIGHBORS_PRUNE, p, radii);
    }
    template <Kernel K = Kernel::cube, class P, class V, class = std::enable_if_t<!std::is_arithmetic<V>::value>>
    std::vector<size_t> neighbors(const P& p, const V& radii) const {
        return oneAxes(K, OCT_NEIGHBORS, p, radii);
    }
    template <Kernel K = Kernel::cube, class P, class V, class = std::enable_if_t<!std::is_arithmetic<V>::value>>
    NeighborSet neighborsStruct(const P& p, const V& radii) const {
        static_assert(K == Kernel::square || K == Kernel::cube, "per-axis radii take the square or cube kernel");
        const double c[3] = {p.getX(), p.getY(), p.getZ()};
        const double r[3] = {radii.getX(), radii.getY(), radii.getZ()};
        std::vector<uint64_t> offs(2), npts(1);
        uint64_t total = 0;
        int st = oct_struct_search_axes(cloud_, static_cast<int>(K), c, 1, r, 0, offs.data(), nullptr, 0, &total,
                                        npts.data(), 0);
        if (st != OCT_OK && st != OCT_ERR_CAPACITY) detail::check(st, cloud_, "oct_struct_search_axes");
        std::vector<uint32_t> pairs(2 * total);
        if (total)
            detail::check(oct_struct_search_axes(cloud_, static_cast<int>(K), c, 1, r, 0, offs.data(), pairs.data(),
                                                 total, &total, npts.data(), 0),
                          cloud_, "oct_struct_search_axes");
        NeighborSet out;
        for (uint64_t j = 0; j < total; ++j) out.ranges.emplace_back(pairs[2 * j], pairs[2 * j + 1]);
        out.numberOfPoints = npts[0];
        return out;
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

    // batched Vector-radii search: radii_xyz nq x 3 (per_query) or one (x, y, z)
    void radiusBatchAxes(Kernel k, int algo, const double* centers, size_t nq, const double* radii_xyz,
                         bool per_query, std::vector<uint64_t>& offsets, std::vector<uint32_t>& idx) const {
        offsets.assign(nq + 1, 0);
        uint64_t total = 0;
        int st = oct_radius_search_axes(cloud_, static_cast<int>(k), algo, centers, nq, radii_xyz, per_query ? 1 : 0,
                                        offsets.data(), nullptr, 0, &total, 0);
        if (st != OCT_OK && st != OCT_ERR_CAPACITY) detail::check(st, cloud_, "oct_radius_search_axes");
        idx.assign(total, 0);
        if (total)
            detail::check(oct_radius_search_axes(cloud_, static_cast<int>(k), algo, centers, nq, radii_xyz,
                                                 per_query ? 1 : 0, offsets.data(), idx.data(), total, &total, 0),
                          cloud_, "oct_radius_search_axes");
    }

private:
    template <class P, class V>
    std::vector<size_t> oneAxes(Kernel k, int algo, const P& p, const V& radii) const {
        if (k != Kernel::square && k != Kernel::cube)
            throw Error(OCT_ERR_INVALID_ARG, "per-axis radii take the square or cube kernel");
        const double c[3] = {p.getX(), p.getY(), p.getZ()};
        const double r[3] = {radii.getX(), radii.getY(), radii.getZ()};
        std::vector<uint64_t> offs;
        std::vector<uint32_t> idx;
        radiusBatchAxes(k, algo, c, 1, r, false, offs, idx);
        return std::vector<size_t>(idx.begin(), idx.end());
    }

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
