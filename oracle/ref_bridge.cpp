// Test infrastructure: a C-ABI bridge over the UNMODIFIED reference implementation
// (derivada/octrees-benchmark), compiled from the reference headers by
// oracle/Makefile into oracle/_ref/libref_octree.so.  Used only by tests/, by
// the golden-fixture script and by bench.py's CPU baseline; never by the product.
//
// Everything here calls the reference's own code path:
//   PointEncoder::sortPoints          inc/encoding/point_encoder.hpp:484-503
//   LinearOctree<PointsAoS> ctor      inc/structures/linear_octree.hpp:614-623
//   neighbors / neighborsPrune / neighborsStruct / knn
//                                     inc/structures/linear_octree.hpp:695-942,1038-1087
// The OpenMP query loops follow inc/benchmarking/neighbor_benchmarks.hpp:502-568.
#include <omp.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <optional>
#include <vector>

#include "benchmarking/search_set.hpp"
#include "encoding/point_encoder_factory.hpp"
#include "structures/linear_octree.hpp"

using PointEncoding::PointEncoder;
using RefKey = PointEncoding::key_t;

namespace {

// Derived class only to read the protected arrays of the built tree.
struct ExposedOctree : public LinearOctree<PointsAoS> {
    using LinearOctree<PointsAoS>::LinearOctree;
    uint32_t n_leaf() const { return nLeaf; }
    uint32_t n_internal() const { return nInternal; }
    uint32_t n_total() const { return nTotal; }
    uint32_t max_depth_seen() const { return maxDepthSeen; }
    const std::vector<uint32_t>& offs() const { return offsets; }
    const std::vector<std::pair<size_t, size_t>>& ranges() const { return internalRanges; }
    const std::vector<Point>& ctrs() const { return centers; }
    const std::vector<Vector>& radii() const { return precomputedRadii; }
    const double* half_lengths() const { return halfLengths; }
};

struct RefCloud {
    PointsAoS points;
    std::vector<RefKey> codes;
    Box box;
    PointEncoder* enc = nullptr;
    std::unique_ptr<ExposedOctree> tree;
    // last radius-search results
    std::vector<std::vector<size_t>> res_idx;
    std::vector<std::vector<std::pair<size_t, size_t>>> res_ranges;
    double t_sort = 0, t_build = 0, t_bbox = 0, t_encode = 0, t_radix = 0;
};

void set_threads(int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    // neighbor_benchmarks.hpp uses schedule(runtime); main.cpp:275 sets it to dynamic
    omp_set_schedule(omp_sched_dynamic, 0);
}

template <Kernel_t K>
void radius_one(const ExposedOctree& t, int algo, const Point& c, double r, std::vector<size_t>& idx,
                std::vector<std::pair<size_t, size_t>>& rng) {
    if (algo == 1) {
        idx = t.neighbors<K>(c, r);
    } else if (algo == 2) {
        idx = t.neighborsPrune<K>(c, r);
    } else {
        auto s = t.neighborsStruct<K>(c, r);
        rng = s.ranges;
        idx.clear();
        idx.reserve(s.numberOfPoints);
        for (auto& pr : s.ranges)
            for (size_t i = pr.first; i < pr.second; ++i) idx.push_back(i);
    }
}

void radius_dispatch(const ExposedOctree& t, int kernel, int algo, const Point& c, double r,
                     std::vector<size_t>& idx, std::vector<std::pair<size_t, size_t>>& rng) {
    switch (kernel) {
        case 0: radius_one<Kernel_t::circle>(t, algo, c, r, idx, rng); break;
        case 1: radius_one<Kernel_t::sphere>(t, algo, c, r, idx, rng); break;
        case 2: radius_one<Kernel_t::square>(t, algo, c, r, idx, rng); break;
        default: radius_one<Kernel_t::cube>(t, algo, c, r, idx, rng); break;
    }
}

template <Kernel_t K>
size_t count_one(const ExposedOctree& t, int algo, const Point& c, double r) {
    if (algo == 1) return t.neighbors<K>(c, r).size();
    if (algo == 2) return t.neighborsPrune<K>(c, r).size();
    return t.neighborsStruct<K>(c, r).size();
}

// neighborsApprox through the reference's public overload (linear_octree.hpp:1089-1093),
// which passes the tolerance percentage on as the precision level
template <Kernel_t K>
void approx_one(const ExposedOctree& t, const Point& c, double r, double tol, bool upper,
                std::vector<std::pair<size_t, size_t>>& rng) {
    auto s = t.neighborsApprox<K>(c, r, tol, upper);
    rng = s.ranges;
}

void approx_dispatch(const ExposedOctree& t, int kernel, const Point& c, double r, double tol, bool upper,
                     std::vector<std::pair<size_t, size_t>>& rng) {
    switch (kernel) {
        case 0: approx_one<Kernel_t::circle>(t, c, r, tol, upper, rng); break;
        case 1: approx_one<Kernel_t::sphere>(t, c, r, tol, upper, rng); break;
        case 2: approx_one<Kernel_t::square>(t, c, r, tol, upper, rng); break;
        default: approx_one<Kernel_t::cube>(t, c, r, tol, upper, rng); break;
    }
}

size_t count_dispatch(const ExposedOctree& t, int kernel, int algo, const Point& c, double r) {
    switch (kernel) {
        case 0: return count_one<Kernel_t::circle>(t, algo, c, r);
        case 1: return count_one<Kernel_t::sphere>(t, algo, c, r);
        case 2: return count_one<Kernel_t::square>(t, algo, c, r);
        default: return count_one<Kernel_t::cube>(t, algo, c, r);
    }
}

template <Kernel_t K>
void axes_one(const ExposedOctree& t, int algo, const Point& c, const Vector& r, std::vector<size_t>& idx,
              std::vector<std::pair<size_t, size_t>>& rng) {
    if (algo == 1) {
        idx = t.neighbors<K>(c, r);
    } else if (algo == 2) {
        idx = t.neighborsPrune<K>(c, r);
    } else {
        auto s = t.neighborsStruct<K>(c, r);
        rng = s.ranges;
        idx.clear();
        for (auto& pr : s.ranges)
            for (size_t i = pr.first; i < pr.second; ++i) idx.push_back(i);
    }
}

}  // namespace

extern "C" {

// Sort (bbox + encode + radix sort) and build the reference octree over an
// AoS xyz array.  Point ids are the input positions 0..n-1.
void* refo_build(int encoder, const double* xyz, uint64_t n, uint64_t max_leaf, int threads) {
    set_threads(threads);
    auto* rc = new RefCloud();
    rc->points = PointsAoS(0);
    for (uint64_t i = 0; i < n; ++i) rc->points.push_back(Point((size_t)i, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
    mainOptions.maxPointsLeaf = (size_t)max_leaf;
    mainOptions.containerType = ContainerType::AoS;
    rc->enc = &PointEncoding::getEncoder((EncoderType)encoder);
    std::optional<std::vector<PointMetadata>> meta = std::nullopt;
    auto elog = std::make_shared<EncodingLog>();
    auto t0 = std::chrono::steady_clock::now();
    auto [codes, box] = rc->enc->sortPoints(rc->points, meta, elog);
    auto t1 = std::chrono::steady_clock::now();
    rc->codes = std::move(codes);
    rc->box = box;
    rc->tree = std::make_unique<ExposedOctree>(rc->points, rc->codes, rc->box, *rc->enc);
    auto t2 = std::chrono::steady_clock::now();
    rc->t_sort = std::chrono::duration<double>(t1 - t0).count();
    rc->t_build = std::chrono::duration<double>(t2 - t1).count();
    rc->t_bbox = elog->boundingBoxTime;
    rc->t_encode = elog->encodingTime;
    rc->t_radix = elog->sortingTime;
    return rc;
}

void refo_free(void* h) { delete static_cast<RefCloud*>(h); }

// out: n, nLeaf, nInternal, nTotal, maxDepthSeen
void refo_info(void* h, uint64_t* out) {
    auto* rc = static_cast<RefCloud*>(h);
    out[0] = rc->points.size();
    out[1] = rc->tree->n_leaf();
    out[2] = rc->tree->n_internal();
    out[3] = rc->tree->n_total();
    out[4] = rc->tree->max_depth_seen();
}

// out: sortPoints+bbox seconds, octree ctor seconds, bbox, encode, radix sort
void refo_times(void* h, double* out) {
    auto* rc = static_cast<RefCloud*>(h);
    out[0] = rc->t_sort;
    out[1] = rc->t_build;
    out[2] = rc->t_bbox;
    out[3] = rc->t_encode;
    out[4] = rc->t_radix;
}

// out: center xyz, radii xyz, min xyz, max xyz of the Box returned by sortPoints
void refo_box(void* h, double* out) {
    auto* rc = static_cast<RefCloud*>(h);
    const Box& b = rc->box;
    out[0] = b.center().getX(); out[1] = b.center().getY(); out[2] = b.center().getZ();
    out[3] = b.radii().getX();  out[4] = b.radii().getY();  out[5] = b.radii().getZ();
    out[6] = b.minX(); out[7] = b.minY(); out[8] = b.minZ();
    out[9] = b.maxX(); out[10] = b.maxY(); out[11] = b.maxZ();
}

// Sorted cloud: xyz (n x 3), original ids, SFC keys
void refo_points(void* h, double* xyz, uint64_t* ids, uint64_t* keys) {
    auto* rc = static_cast<RefCloud*>(h);
    size_t n = rc->points.size();
    for (size_t i = 0; i < n; ++i) {
        const Point& p = rc->points[i];
        if (xyz) { xyz[3 * i] = p.getX(); xyz[3 * i + 1] = p.getY(); xyz[3 * i + 2] = p.getZ(); }
        if (ids) ids[i] = p.id();
        if (keys) keys[i] = rc->codes[i];
    }
}

// Tree arrays: offsets (nTotal+1), ranges (nTotal x 2), centers (nTotal x 3),
// per-level radii (22 x 3), halfLengths (3)
void refo_tree(void* h, uint32_t* offsets, uint64_t* ranges, double* centers, double* radii, double* half) {
    auto* rc = static_cast<RefCloud*>(h);
    const auto& t = *rc->tree;
    uint32_t nt = t.n_total();
    for (uint32_t i = 0; i <= nt; ++i) offsets[i] = t.offs()[i];
    for (uint32_t i = 0; i < nt; ++i) {
        ranges[2 * i] = t.ranges()[i].first;
        ranges[2 * i + 1] = t.ranges()[i].second;
        centers[3 * i] = t.ctrs()[i].getX();
        centers[3 * i + 1] = t.ctrs()[i].getY();
        centers[3 * i + 2] = t.ctrs()[i].getZ();
    }
    for (size_t l = 0; l < t.radii().size(); ++l) {
        radii[3 * l] = t.radii()[l].getX();
        radii[3 * l + 1] = t.radii()[l].getY();
        radii[3 * l + 2] = t.radii()[l].getZ();
    }
    for (int a = 0; a < 3; ++a) half[a] = t.half_lengths()[a];
}

// Radius search over nq centers (xyz AoS) with per-query radii.  kernel follows
// Kernel_t (0 circle, 1 sphere, 2 square, 3 cube); algo 1 neighbors,
// 2 neighborsPrune, 3 neighborsStruct.  Returns the total number of indices;
// the results stay in the handle until refo_radius_fetch.
uint64_t refo_radius(void* h, int kernel, int algo, const double* centers, uint64_t nq, const double* radii,
                     int threads) {
    set_threads(threads);
    auto* rc = static_cast<RefCloud*>(h);
    rc->res_idx.assign(nq, {});
    rc->res_ranges.assign(nq, {});
    #pragma omp parallel for schedule(runtime)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        Point c(centers[3 * q], centers[3 * q + 1], centers[3 * q + 2]);
        radius_dispatch(*rc->tree, kernel, algo, c, radii[q], rc->res_idx[q], rc->res_ranges[q]);
    }
    uint64_t total = 0;
    for (auto& v : rc->res_idx) total += v.size();
    return total;
}

// offsets (nq+1), idx (total) in the reference's own emission order
void refo_radius_fetch(void* h, uint64_t* offsets, uint64_t* idx) {
    auto* rc = static_cast<RefCloud*>(h);
    uint64_t o = 0;
    for (size_t q = 0; q < rc->res_idx.size(); ++q) {
        offsets[q] = o;
        for (size_t v : rc->res_idx[q]) idx[o++] = v;
    }
    offsets[rc->res_idx.size()] = o;
}

// The Vector-radii overloads (linear_octree.hpp:1044-1048, 1056-1060, 1069-1074) over nq centers with
// per-query (rx, ry, rz) radii (nq x 3); kernel 2 square or 3 cube, algo as refo_radius.  Results stay
// in the handle like refo_radius's (refo_radius_fetch, refo_struct_ranges_fetch).
uint64_t refo_radius_axes(void* h, int kernel, int algo, const double* centers, uint64_t nq, const double* radii3,
                          int threads) {
    set_threads(threads);
    auto* rc = static_cast<RefCloud*>(h);
    rc->res_idx.assign(nq, {});
    rc->res_ranges.assign(nq, {});
    #pragma omp parallel for schedule(runtime)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        Point c(centers[3 * q], centers[3 * q + 1], centers[3 * q + 2]);
        Vector r(radii3[3 * q], radii3[3 * q + 1], radii3[3 * q + 2]);
        if (kernel == 2) axes_one<Kernel_t::square>(*rc->tree, algo, c, r, rc->res_idx[q], rc->res_ranges[q]);
        else axes_one<Kernel_t::cube>(*rc->tree, algo, c, r, rc->res_idx[q], rc->res_ranges[q]);
    }
    uint64_t total = 0;
    for (auto& v : rc->res_idx) total += v.size();
    return total;
}

// neighborsApprox over nq centers; the ranges stay in the handle (refo_struct_ranges_fetch).
// Returns the number of ranges.
uint64_t refo_approx(void* h, int kernel, const double* centers, uint64_t nq, const double* radii, double tol,
                     int upper, int threads) {
    set_threads(threads);
    auto* rc = static_cast<RefCloud*>(h);
    rc->res_idx.assign(nq, {});
    rc->res_ranges.assign(nq, {});
    #pragma omp parallel for schedule(runtime)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        Point c(centers[3 * q], centers[3 * q + 1], centers[3 * q + 2]);
        approx_dispatch(*rc->tree, kernel, c, radii[q], tol, upper != 0, rc->res_ranges[q]);
    }
    uint64_t total = 0;
    for (auto& v : rc->res_ranges) total += v.size();
    return total;
}

uint64_t refo_struct_range_total(void* h) {
    auto* rc = static_cast<RefCloud*>(h);
    uint64_t t = 0;
    for (auto& v : rc->res_ranges) t += v.size();
    return t;
}

// ranges of the last neighborsStruct call: offsets (nq+1) and (first,last) pairs
void refo_struct_ranges_fetch(void* h, uint64_t* offsets, uint64_t* pairs) {
    auto* rc = static_cast<RefCloud*>(h);
    uint64_t o = 0;
    for (size_t q = 0; q < rc->res_ranges.size(); ++q) {
        offsets[q] = o;
        for (auto& pr : rc->res_ranges[q]) { pairs[2 * o] = pr.first; pairs[2 * o + 1] = pr.second; ++o; }
    }
    offsets[rc->res_ranges.size()] = o;
}

// kNN: idx/d2 are nq x k; counts[q] = number of valid entries (min(n, k)).
void refo_knn(void* h, const double* centers, uint64_t nq, uint64_t k, uint64_t* idx, double* d2, uint64_t* counts,
              int threads) {
    set_threads(threads);
    auto* rc = static_cast<RefCloud*>(h);
    #pragma omp parallel for schedule(runtime)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        Point c(centers[3 * q], centers[3 * q + 1], centers[3 * q + 2]);
        std::vector<size_t> ii(k, (size_t)-1);
        std::vector<double> dd(k, -1.0);
        size_t got = rc->tree->knn(c, k, ii, dd);
        counts[q] = got;
        for (uint64_t j = 0; j < k; ++j) { idx[q * k + j] = ii[j]; d2[q * k + j] = dd[j]; }
    }
}

// splitmix64's output function: the per-index term of the set hash below.
static inline uint64_t mix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Radius search over nq centers with one radius, kept as a per-query count and
// an order-independent hash of the neighbour index set (the sum of mix64 of
// every index, modulo 2^64), so that sweeps over whole clouds need no result
// storage.  Same kernels and algos as refo_radius.
void refo_radius_hash(void* h, int kernel, int algo, const double* centers, uint64_t nq, double radius, int threads,
                      uint64_t* counts, uint64_t* hashes) {
    set_threads(threads);
    auto* rc = static_cast<RefCloud*>(h);
    #pragma omp parallel
    {
        std::vector<size_t> idx;
        std::vector<std::pair<size_t, size_t>> rng;
        #pragma omp for schedule(runtime)
        for (int64_t q = 0; q < (int64_t)nq; ++q) {
            Point c(centers[3 * q], centers[3 * q + 1], centers[3 * q + 2]);
            radius_dispatch(*rc->tree, kernel, algo, c, radius, idx, rng);
            uint64_t s = 0;
            for (size_t v : idx) s += mix64((uint64_t)v);
            counts[q] = idx.size();
            hashes[q] = s;
        }
    }
}

// ---- timed loops for the CPU baseline (steady_clock wall time, seconds) ----

double refo_time_radius(void* h, int kernel, int algo, const double* centers, uint64_t nq, double radius,
                        int threads, uint64_t* total_out) {
    set_threads(threads);
    auto* rc = static_cast<RefCloud*>(h);
    uint64_t total = 0;
    auto t0 = std::chrono::steady_clock::now();
    #pragma omp parallel for schedule(runtime) reduction(+ : total)
    for (int64_t q = 0; q < (int64_t)nq; ++q) {
        Point c(centers[3 * q], centers[3 * q + 1], centers[3 * q + 2]);
        total += count_dispatch(*rc->tree, kernel, algo, c, radius);
    }
    auto t1 = std::chrono::steady_clock::now();
    if (total_out) *total_out = total;
    return std::chrono::duration<double>(t1 - t0).count();
}

double refo_time_knn(void* h, const double* centers, uint64_t nq, uint64_t k, int threads, double* checksum) {
    set_threads(threads);
    auto* rc = static_cast<RefCloud*>(h);
    double acc = 0;
    auto t0 = std::chrono::steady_clock::now();
    #pragma omp parallel reduction(+ : acc)
    {
        std::vector<size_t> ii(k);
        std::vector<double> dd(k);
        #pragma omp for schedule(runtime)
        for (int64_t q = 0; q < (int64_t)nq; ++q) {
            Point c(centers[3 * q], centers[3 * q + 1], centers[3 * q + 2]);
            size_t got = rc->tree->knn(c, k, ii, dd);
            if (got) acc += dd[got - 1];
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    if (checksum) *checksum = acc;
    return std::chrono::duration<double>(t1 - t0).count();
}

int refo_max_threads() { return omp_get_max_threads(); }

// The reference's SearchSet (inc/benchmarking/search_set.hpp:23-44): `repeats`
// rows of n centre indices into a cloud of cloud_size points, random
// (mt19937 seeded 42, uniform_int_distribution) or a sequential slice.
// out: repeats x n' indices, n' = cloud_size when `all` is set, else n.
void refo_search_set(uint64_t n, uint64_t cloud_size, int sequential, int all, uint64_t repeats, uint64_t* out) {
    mainOptions.repeats = (size_t)repeats;
    SearchSet s((size_t)n, (size_t)cloud_size, sequential != 0, all != 0);
    uint64_t o = 0;
    for (const auto& row : s.searchPoints)
        for (size_t v : row) out[o++] = v;
}

// PointEncoder::getAnchorCoords (point_encoder.hpp:37-49) on one axis value,
// with the box given by its center and radii (Box(center, radii), box.hpp:17).
uint64_t refo_anchor(double p, double c, double r) {
    Box b(Point(c, c, c), Vector(r, r, r));
    PointEncoding::coords_t x, y, z;
    PointEncoding::getEncoder(EncoderType::MORTON_ENCODER_3D).getAnchorCoords(Point(p, p, p), b, x, y, z);
    return (uint64_t)x;
}

uint64_t refo_encode(int encoder, uint64_t x, uint64_t y, uint64_t z) {
    return PointEncoding::getEncoder((EncoderType)encoder).encode(x, y, z);
}

void refo_decode(int encoder, uint64_t key, uint64_t* xyz) {
    PointEncoding::coords_t x, y, z;
    PointEncoding::getEncoder((EncoderType)encoder).decode(key, x, y, z);
    xyz[0] = x; xyz[1] = y; xyz[2] = z;
}

}  // extern "C"
