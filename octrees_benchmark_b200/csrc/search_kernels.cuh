// Search-kernel predicates on the device: sphere, cube, square, circle.
// Each is the reference's arithmetic in the reference's operation order, with
// round-to-nearest FP64 ops and no contraction, so every decision is bitwise
// the reference's.
#pragma once
#include "oct_common.cuh"

namespace octb {

// Kernel_t values (inc/main_options.hpp:97-103)
enum KernelType : int { kCircle = 0, kSphere = 1, kSquare = 2, kCube = 3 };
// SearchAlgo order for the three linear-octree radius searches
enum Algo : int { kNeighbors = 1, kPrune = 2, kStruct = 3 };
enum Judgement : int { kOutside = 0, kOverlap = 1, kInside = 2 };

struct SearchKernel {
    double c[3];
    double r, r2;
    double bmin[3], bmax[3];

    // KernelAbstract(center, radius) + makeBox (kernel_abstract.hpp:32-45);
    // radiusSq_ = radius * radius (kernel_3d.hpp:164, kernel_2d.hpp:49)
    __device__ __forceinline__ void init(double cx, double cy, double cz, double radius) {
        c[0] = cx; c[1] = cy; c[2] = cz;
        r = radius;
        r2 = dmul(radius, radius);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            bmin[a] = dsub(c[a], radius);
            bmax[a] = dadd(c[a], radius);
        }
    }

    // KernelAbstract(center, Vector radii) + makeBox (kernel_abstract.hpp:36, 41-45): the box
    // center -/+ radii per axis; only the cube and square kernels take it (kernel_factory.hpp:33-41),
    // and they read nothing but the box
    __device__ __forceinline__ void init_axes(double cx, double cy, double cz, const double* rad) {
        c[0] = cx; c[1] = cy; c[2] = cz;
        r = rad[0];
        r2 = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            bmin[a] = dsub(c[a], rad[a]);
            bmax[a] = dadd(c[a], rad[a]);
        }
    }
};

// isInside: sphere strict < (kernel_3d.hpp:168-179), circle <= (kernel_2d.hpp:53-63),
// cube / square closed intervals via onInterval (kernel_3d.hpp:273-283,
// kernel_2d.hpp:153-162, util.hpp:134-137)
template <int KT>
__device__ __forceinline__ bool is_inside(const SearchKernel& k, double px, double py, double pz) {
    if constexpr (KT == kSphere) {
        return dsq3(dsub(px, k.c[0]), dsub(py, k.c[1]), dsub(pz, k.c[2])) < k.r2;
    } else if constexpr (KT == kCircle) {
        return dsq2(dsub(px, k.c[0]), dsub(py, k.c[1])) <= k.r2;
    } else if constexpr (KT == kCube) {
        return px >= k.bmin[0] && px <= k.bmax[0] && py >= k.bmin[1] && py <= k.bmax[1] && pz >= k.bmin[2] &&
               pz <= k.bmax[2];
    } else {
        return px >= k.bmin[0] && px <= k.bmax[0] && py >= k.bmin[1] && py <= k.bmax[1];
    }
}

// boxIntersect(octantCenter, Vector octantRadii): sphere kernel_3d.hpp:222-264,
// cube 318-343, circle kernel_2d.hpp:107-144, square 195-218
template <int KT>
__device__ __forceinline__ int box_intersect(const SearchKernel& k, const double* oc, const double* orr) {
    if constexpr (KT == kSphere || KT == kCircle) {
        constexpr int D = (KT == kSphere) ? 3 : 2;
        double d[3], cc[3];
        bool out = false;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            d[a] = fabs(dsub(k.c[a], oc[a]));
            out = out || (d[a] > dadd(k.r, orr[a]));
        }
        if (out) return kOutside;
#pragma unroll
        for (int a = 0; a < D; ++a) cc[a] = dadd(d[a], orr[a]);
        const double far2 = (D == 3) ? dsq3(cc[0], cc[1], cc[2]) : dsq2(cc[0], cc[1]);
        if (far2 <= k.r2) return kInside;
        int ninside = 0;
#pragma unroll
        for (int a = 0; a < D; ++a) ninside += (d[a] < orr[a]);
        if (ninside > 1) return kOverlap;
#pragma unroll
        for (int a = 0; a < D; ++a) d[a] = smax(dsub(d[a], orr[a]), 0.0);
        const double near2 = (D == 3) ? dsq3(d[0], d[1], d[2]) : dsq2(d[0], d[1]);
        return (near2 <= k.r2) ? kOverlap : kOutside;
    } else {
        constexpr int D = (KT == kCube) ? 3 : 2;
        double hi[3], lo[3];
#pragma unroll
        for (int a = 0; a < D; ++a) {
            hi[a] = dadd(oc[a], orr[a]);
            lo[a] = dsub(oc[a], orr[a]);
        }
        bool out = false, in = true;
#pragma unroll
        for (int a = 0; a < D; ++a) out = out || (hi[a] < k.bmin[a]);
#pragma unroll
        for (int a = 0; a < D; ++a) out = out || (lo[a] > k.bmax[a]);
        if (out) return kOutside;
#pragma unroll
        for (int a = 0; a < D; ++a) in = in && (hi[a] <= k.bmax[a]);
#pragma unroll
        for (int a = 0; a < D; ++a) in = in && (lo[a] >= k.bmin[a]);
        return in ? kInside : kOverlap;
    }
}

// boxOverlap(center, Vector radii): Kernel3D (kernel_3d.hpp:141-156) for sphere
// and cube, Kernel2D (kernel_2d.hpp:29-41) for circle and square
template <int KT>
__device__ __forceinline__ bool box_overlap(const SearchKernel& k, const double* oc, const double* orr) {
    constexpr int D = (KT == kSphere || KT == kCube) ? 3 : 2;
    bool out = false;
#pragma unroll
    for (int a = 0; a < D; ++a) out = out || (dadd(oc[a], orr[a]) < k.bmin[a]);
#pragma unroll
    for (int a = 0; a < D; ++a) out = out || (dsub(oc[a], orr[a]) > k.bmax[a]);
    return !out;
}

// kNN distances (linear_octree.hpp:844-878): point-point and the clamp-to-box
// point-octant lower bound.
__device__ __forceinline__ double dist_pp(double px, double py, double pz, double qx, double qy, double qz) {
    return dsq3(dsub(px, qx), dsub(py, qy), dsub(pz, qz));
}
__device__ __forceinline__ double dist_po(const double* p, const double* oc, const double* orr) {
    double d[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double lo = dsub(oc[a], orr[a]);
        const double hi = dadd(oc[a], orr[a]);
        const double c = smax(lo, smin(p[a], hi));
        d[a] = dsub(p[a], c);
    }
    return dsq3(d[0], d[1], d[2]);
}

}  // namespace octb
