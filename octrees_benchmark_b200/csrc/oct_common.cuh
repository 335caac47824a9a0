// Shared device-side definitions for the B200 linear-octree neighbour search.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace octb {

constexpr uint32_t kMaxDepth = 21;                       // 3 bits per level, 63-bit keys
constexpr uint64_t kUpperBound = 0x8000000000000000ull;  // first key past every valid key
constexpr uint64_t kMaxCoord = (1ull << kMaxDepth) - 1;

// Device error word bits (OR-ed into Cloud::d_err by kernels; read by the host).
enum ErrBits : uint32_t {
    kErrSpinLimit = 1u << 0,      // a bounded wait gave up
    kErrStackOverflow = 1u << 1,  // traversal stack bound reached
    kErrNodeCapacity = 1u << 2,   // octree node arrays too small (host re-runs larger)
    kErrOutputCapacity = 1u << 3, // result buffer smaller than the counted results
    kErrBadInput = 1u << 4,       // invalid query (e.g. k larger than supported)
    kErrChunkCapacity = 1u << 5,  // one-pass radius: result chunk pool too small (counts still exact)
};

// Bounded spin: every wait in this library gives up after this many polls.
constexpr uint32_t kSpinLimit = 1u << 26;

__device__ __forceinline__ void set_err(uint32_t* err, uint32_t bits) { atomicOr(err, bits); }

// splitmix64's output function: the term of one neighbour index in the
// order-independent set hash of oct_radius_hash (the sum of the terms mod 2^64).
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---- exact FP64 helpers: every decision uses round-to-nearest ops with no
// contraction, matching the reference's x86 build (no -mfma). ----
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsq3(double a, double b, double c) {
    return dadd(dadd(dmul(a, a), dmul(b, b)), dmul(c, c));
}
__device__ __forceinline__ double dsq2(double a, double b) { return dadd(dmul(a, a), dmul(b, b)); }
// std::max(a, b) / std::min(a, b) semantics (first argument wins on ties and NaN)
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }

// Box of a cloud, as PointEncoder::sortPoints builds it: Box(center, radii).
struct BoxD {
    double center[3];
    double radii[3];
    double min[3];
    double max[3];
};

// Per-level node radii and the half lengths of the finest cell.
struct LevelGeom {
    double radii[kMaxDepth + 1][3];
    double half[3];
};

}  // namespace octb
