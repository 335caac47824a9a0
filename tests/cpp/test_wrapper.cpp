// The reference's own GoogleTest cases (tests/structures/test_octree.cpp,
// test_octree_advanced.cpp, tests/integration/test_complex.cpp,
// tests/encoding/test_encoders.cpp), restated against the C++ drop-in
// include/linear_octree_gpu.hpp on the GPU.  The point and container types
// below have the members the reference's Point / PointsAoS expose and the
// wrapper uses.  Built and run by tests/test_gpu_cpp_wrapper.py.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <optional>
#include <random>
#include <vector>

#include "linear_octree_gpu.hpp"

namespace {

int fails = 0;
#define EXPECT(c)                                                             \
    do {                                                                      \
        if (!(c)) {                                                           \
            std::fprintf(stderr, "FAIL %s:%d  %s\n", __FILE__, __LINE__, #c); \
            ++fails;                                                          \
        }                                                                     \
    } while (0)

struct Point {
    double x_ = 0, y_ = 0, z_ = 0;
    size_t id_ = 0;
    Point() = default;
    Point(double x, double y, double z, size_t id = 0) : x_(x), y_(y), z_(z), id_(id) {}
    double getX() const { return x_; }
    double getY() const { return y_; }
    double getZ() const { return z_; }
    size_t id() const { return id_; }
};

struct PointsAoS {
    std::vector<Point> data;
    size_t size() const { return data.size(); }
    const Point& operator[](size_t i) const { return data[i]; }
    Point& operator[](size_t i) { return data[i]; }
    void set(size_t i, const Point& p) { data[i] = p; }
    void push_back(const Point& p) { data.push_back(Point(p.x_, p.y_, p.z_, data.size())); }
};

using octree_b200::Encoder;
using octree_b200::Kernel;
using Oct = octree_b200::LinearOctree<PointsAoS>;

double sq(const Point& a, const Point& b) {
    const double dx = a.getX() - b.getX(), dy = a.getY() - b.getY(), dz = a.getZ() - b.getZ();
    return dx * dx + dy * dy + dz * dz;
}

void test_octree_cpp() {  // test_octree.cpp:17-80
    PointsAoS pts;
    for (auto p : {Point(0, 0, 0), Point(0.1, 0, 0), Point(0, 0.1, 0), Point(10, 10, 10), Point(10.1, 10, 10),
                   Point(10, 10.1, 10), Point(5, 5, 5), Point(5, 5, 5.1)})
        pts.push_back(p);
    std::vector<uint64_t> codes;
    Oct oct(pts, codes, Encoder::morton);
    EXPECT(std::is_sorted(codes.begin(), codes.end()));
    std::vector<size_t> idx(2);
    std::vector<double> d(2);
    EXPECT(oct.knn(Point(9.9, 9.9, 9.9), 2, idx, d) == 2);
    EXPECT(std::fabs(d[0] - 0.03) < 1e-4);
    EXPECT(pts[idx[0]].getX() > 9.0);
    auto r = oct.neighborsPrune<Kernel::square>(Point(5, 5, 5), 0.25);
    EXPECT(r.size() == 2);
    std::vector<double> zs;
    for (size_t i : r) zs.push_back(pts[i].getZ());
    std::sort(zs.begin(), zs.end());
    EXPECT(zs.size() == 2 && zs[0] == 5.0 && zs[1] == 5.1);
}

void test_octree_advanced_cpp() {  // test_octree_advanced.cpp:33-131
    {
        PointsAoS pts;  // empty cloud
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, Encoder::morton);
        EXPECT(oct.neighborsPrune<Kernel::square>(Point(0, 0, 0), 1.0).empty());
        std::vector<size_t> i(1);
        std::vector<double> d(1);
        EXPECT(oct.knn(Point(0, 0, 0), 1, i, d) == 0);
    }
    {
        PointsAoS pts;  // duplicates
        for (auto p : {Point(1, 1, 1), Point(1, 1, 1), Point(2, 2, 2)}) pts.push_back(p);
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, Encoder::morton);
        std::vector<size_t> i(5);
        std::vector<double> d(5);
        EXPECT(oct.knn(Point(1, 1, 1), 5, i, d) == 3);
        EXPECT(std::fabs(d[0]) < 1e-9 && std::fabs(d[1]) < 1e-9);
        EXPECT(std::fabs(d[2] - sq(Point(1, 1, 1), pts[i[2]])) < 1e-9);
    }
    {
        PointsAoS pts;  // zero radius
        for (auto p : {Point(0, 0, 0), Point(0, 0, 0), Point(1, 1, 1)}) pts.push_back(p);
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, Encoder::morton);
        auto r = oct.neighborsPrune<Kernel::square>(Point(0, 0, 0), 0.0);
        EXPECT(r.size() == 2);
        for (size_t i : r) EXPECT(sq(pts[i], Point(0, 0, 0)) == 0.0);
    }
    {
        PointsAoS pts;  // boundary
        for (auto p : {Point(0, 0, 0), Point(10, 10, 10), Point(5, 5, 5)}) pts.push_back(p);
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, Encoder::morton);
        auto r = oct.neighborsPrune<Kernel::square>(Point(10, 10, 10), 0.0);
        EXPECT(r.size() == 1 && sq(pts[r[0]], Point(10, 10, 10)) == 0.0);
        EXPECT(oct.neighborsPrune<Kernel::square>(Point(10.1, 10.1, 10.1), 0.01).empty());
    }
    {
        PointsAoS pts;  // sphere
        for (auto p : {Point(1, 1, 1), Point(2, 0, 0)}) pts.push_back(p);
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, Encoder::morton);
        EXPECT(oct.neighborsPrune<Kernel::sphere>(Point(0, 0, 0), 1.5).empty());
        EXPECT(oct.neighborsPrune<Kernel::sphere>(Point(0, 0, 0), 2.5).size() == 2);
    }
    {
        PointsAoS pts;  // cube
        for (auto p : {Point(1, 1, 1), Point(2, 2, 2)}) pts.push_back(p);
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, Encoder::morton);
        auto r = oct.neighborsPrune<Kernel::cube>(Point(0, 0, 0), 1.5);
        EXPECT(r.size() == 1 && pts[r[0]].getX() == 1.0);
    }
}

size_t brute(const PointsAoS& pts, const Point& c, double r) {  // test_complex.cpp:22-33 (<=)
    size_t n = 0;
    for (size_t i = 0; i < pts.size(); ++i) n += sq(pts[i], c) <= r * r;
    return n;
}

void test_complex_cpp() {  // test_complex.cpp:37-173
    {
        PointsAoS pts;
        for (int i = 0; i < 100; ++i) pts.push_back(Point(i * 0.1, 0, 0));
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, Encoder::morton);
        EXPECT(oct.neighborsPrune<Kernel::sphere>(Point(5, 0, 0), 0.55).size() == brute(pts, Point(5, 0, 0), 0.55));
    }
    {
        PointsAoS pts;
        for (int i = 0; i < 10; ++i)
            for (int j = 0; j < 10; ++j) pts.push_back(Point(i * 0.1, j * 0.1, 0));
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, Encoder::morton);
        EXPECT(oct.neighborsPrune<Kernel::sphere>(Point(0.5, 0.5, 0), 0.2).size() ==
               brute(pts, Point(0.5, 0.5, 0), 0.2));
    }
    {
        const double o = 1e6;
        PointsAoS pts;
        for (auto p : {Point(o, o, o), Point(o + 0.1, o, o), Point(o, o + 0.1, o)}) pts.push_back(p);
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, Encoder::morton);
        EXPECT(oct.neighborsPrune<Kernel::sphere>(Point(o + 0.05, o + 0.05, o), 0.1).size() == 3);
    }
    for (Encoder enc : {Encoder::morton, Encoder::hilbert}) {
        PointsAoS pts;  // KNNConsistency, same generator as the reference test
        std::mt19937 gen(42);
        std::uniform_real_distribution<> dis(0, 10);
        for (int i = 0; i < 500; ++i) pts.push_back(Point(dis(gen), dis(gen), dis(gen)));
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, enc);
        std::vector<size_t> idx(10);
        std::vector<double> d(10);
        oct.knn(Point(5, 5, 5), 10, idx, d);
        for (int i = 1; i < 10; ++i) EXPECT(d[i] >= d[i - 1]);
        for (int i = 0; i < 10; ++i) EXPECT(std::fabs(d[i] - sq(pts[idx[i]], Point(5, 5, 5))) < 1e-7);
        // neighborsStruct covers the same points as neighborsPrune; every variant agrees with brute force (<)
        for (double r : {0.5, 2.0}) {
            auto pr = oct.neighborsPrune<Kernel::sphere>(Point(5, 5, 5), r);
            auto nb = oct.neighbors<Kernel::sphere>(Point(5, 5, 5), r);
            auto st = oct.neighborsStruct<Kernel::sphere>(Point(5, 5, 5), r);
            auto si = st.indices();
            std::sort(pr.begin(), pr.end());
            std::sort(nb.begin(), nb.end());
            std::sort(si.begin(), si.end());
            EXPECT(pr == nb && pr == si && st.size() == pr.size());
            size_t strict = 0;
            for (size_t i = 0; i < pts.size(); ++i) strict += sq(pts[i], Point(5, 5, 5)) < r * r;
            EXPECT(pr.size() == strict);
            // neighborsApprox bounds (the reference's ApproxSearchBounds, test_complex.cpp:115-141):
            // upper >= exact >= lower, at its level (maxDepth / 2 = 10) and at levels that cut
            for (double tol : {10.0, 2.0, 1.0}) {
                auto up = oct.neighborsApprox<Kernel::sphere>(Point(5, 5, 5), r, tol, true);
                auto lo = oct.neighborsApprox<Kernel::sphere>(Point(5, 5, 5), r, tol, false);
                EXPECT(up.size() >= st.size() && lo.size() <= st.size());
            }
        }
        // points were reordered in place, ids travel with them
        std::vector<size_t> ids;
        for (size_t i = 0; i < pts.size(); ++i) ids.push_back(pts[i].id());
        std::sort(ids.begin(), ids.end());
        for (size_t i = 0; i < ids.size(); ++i) EXPECT(ids[i] == i);
        EXPECT(std::is_sorted(codes.begin(), codes.end()));
    }
}

void test_encoders_cpp() {  // test_encoders.cpp:29-64
    for (Encoder enc : {Encoder::morton, Encoder::hilbert}) {
        PointsAoS pts;
        for (auto p : {Point(1, 1, 1), Point(9, 9, 9), Point(5, 5, 5), Point(1, 9, 1)}) pts.push_back(p);
        std::vector<uint64_t> codes;
        Oct oct(pts, codes, enc);
        EXPECT(codes.size() == 4 && pts.size() == 4);
        EXPECT(oct.box().min[0] == 1.0 && oct.box().max[0] == 9.0);
        EXPECT(oct.box().min[1] == 1.0 && oct.box().max[1] == 9.0);
        if (enc == Encoder::morton) {
            EXPECT(pts[0].getX() == 1.0 && pts[0].getY() == 1.0 && pts[0].getZ() == 1.0);
            EXPECT(pts[3].getX() == 9.0 && pts[3].getY() == 9.0 && pts[3].getZ() == 9.0);
        }
    }
}

struct Vec {  // the reference's Vector: per-axis radii
    double x, y, z;
    double getX() const { return x; }
    double getY() const { return y; }
    double getZ() const { return z; }
};

struct Meta {  // stands in for PointMetadata: it travels with its point
    size_t tag;
};

void test_example_cpp() {  // examples/example.cpp:14-47, the same calls in namespace octree_b200
    using namespace octree_b200;
    PointsAoS points;
    points.push_back(Point(1.2, 3.4, 5.6));
    points.push_back(Point(7.8, 9.0, 1.2));
    points.push_back(Point(3.4, 5.6, 7.8));
    points.push_back(Point(9.0, 1.2, 3.4));
    std::optional<std::vector<Meta>> metadata = std::nullopt;
    PointEncoding::MortonEncoder3D enc;
    auto [codes, box] = enc.sortPoints(points, metadata);
    LinearOctree octree(points, codes, box, enc);
    size_t k = 2;
    std::vector<size_t> indexes(k);
    std::vector<double> distances(k);
    Point searchPoint(5.0, 5.0, 5.0);
    EXPECT(octree.knn(searchPoint, k, indexes, distances) == 2);
    for (size_t i = 0; i < k; ++i) EXPECT(std::fabs(distances[i] - sq(points[indexes[i]], searchPoint)) < 1e-12);
    EXPECT(distances[0] <= distances[1]);
}

void test_two_step_equals_one_step_cpp() {
    // sortPoints + LinearOctree(points, codes, box, enc) (with metadata moved along) against the one-step octree
    using namespace octree_b200;
    for (EncoderType et : {MORTON_ENCODER_3D, HILBERT_ENCODER_3D}) {
        PointsAoS a, b;
        std::mt19937 gen(7);
        std::uniform_real_distribution<> dis(0, 50);
        for (int i = 0; i < 3000; ++i) {
            Point p(dis(gen), dis(gen), dis(gen) * 0.2);
            a.push_back(p);
            b.push_back(p);
        }
        std::optional<std::vector<Meta>> meta = std::vector<Meta>();
        for (size_t i = 0; i < a.size(); ++i) meta->push_back(Meta{i});
        mainOptions.maxPointsLeaf = 16;
        auto& enc = PointEncoding::getEncoder(et);
        auto [codes, box] = enc.sortPoints(a, meta);
        LinearOctree two(a, codes, box, enc);
        std::vector<uint64_t> codes1;
        Oct one(b, codes1, et == MORTON_ENCODER_3D ? Encoder::morton : Encoder::hilbert, 16);
        mainOptions.maxPointsLeaf = 128;
        EXPECT(codes == codes1);
        EXPECT(two.nTotal() == one.nTotal() && two.nLeaf() == one.nLeaf());
        for (size_t i = 0; i < a.size(); ++i) EXPECT(a[i].id() == b[i].id() && (*meta)[i].tag == a[i].id());
        for (int q = 0; q < 50; ++q) {
            const Point& c = a[(q * 61) % a.size()];
            auto r1 = two.neighborsPrune<Kernel_t::sphere>(c, 3.0);
            auto r2 = one.neighborsPrune<Kernel_t::sphere>(c, 3.0);
            std::sort(r1.begin(), r1.end());
            std::sort(r2.begin(), r2.end());
            EXPECT(r1 == r2);
            // Vector radii: cube and square against brute force (closed intervals)
            const Vec rv{2.5, 0.7, 1.4};
            auto cu = two.neighborsPrune<Kernel_t::cube>(c, rv);
            auto sqr = two.neighbors<Kernel_t::square>(c, rv);
            auto st = two.neighborsStruct<Kernel_t::cube>(c, rv);
            size_t n3 = 0, n2 = 0;
            for (size_t i = 0; i < a.size(); ++i) {
                const bool in2 = a[i].getX() >= c.getX() - rv.x && a[i].getX() <= c.getX() + rv.x &&
                                 a[i].getY() >= c.getY() - rv.y && a[i].getY() <= c.getY() + rv.y;
                n2 += in2;
                n3 += in2 && a[i].getZ() >= c.getZ() - rv.z && a[i].getZ() <= c.getZ() + rv.z;
            }
            EXPECT(cu.size() == n3 && st.size() == n3 && sqr.size() == n2);
        }
    }
}

}  // namespace

int main() {
    try {
        test_octree_cpp();
        test_octree_advanced_cpp();
        test_complex_cpp();
        test_encoders_cpp();
        test_example_cpp();
        test_two_step_equals_one_step_cpp();
    } catch (const octree_b200::Error& e) {
        std::fprintf(stderr, "octree_b200::Error status %d: %s\n", e.status(), e.what());
        return 2;
    }
    std::printf("%s (%d failures)\n", fails ? "FAILED" : "OK", fails);
    return fails ? 1 : 0;
}
