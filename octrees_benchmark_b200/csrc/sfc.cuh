// Space-filling-curve keys on the device: anchor coordinates, Morton and
// Hilbert 63-bit encode/decode, and the key algebra of the linear octree.
#pragma once
#include "oct_common.cuh"

namespace octb {

// double -> 64-bit unsigned conversion with x86-64 semantics, which is what
// the reference's (coords_t) cast compiles to: values below 2^63 (and NaN,
// which compares unordered) take the signed truncation, whose out-of-range
// result is 0x8000000000000000; values from 2^63 up take (v - 2^63) and an
// xor of the top bit.  The CUDA cast saturates instead, so it is emulated.
__device__ __forceinline__ uint64_t x86_cvt_u64(double v) {
    const double two63 = 9223372036854775808.0;
    if (v != v) return 1ull << 63;
    if (v < two63) {
        if (v <= -two63) return 1ull << 63;
        return (uint64_t)__double2ll_rz(v);
    }
    double w = dsub(v, two63);
    uint64_t s = (w < two63) ? (uint64_t)__double2ll_rz(w) : (1ull << 63);
    return s ^ (1ull << 63);
}

// PointEncoder::getAnchorCoords, one axis (inc/encoding/point_encoder.hpp:37-49):
// x = min((coords_t)(((p - c) + r) / (2 r) * 2^21), 2^21 - 1)
__device__ __forceinline__ uint32_t anchor_coord(double p, double c, double r) {
    double t = ddiv(dadd(dsub(p, c), r), dmul(2.0, r));
    uint64_t u = x86_cvt_u64(dmul(t, 2097152.0));
    return (uint32_t)(u < kMaxCoord ? u : kMaxCoord);
}

// Morton: coordinate bit i goes to key bit 3i (x), 3i+1 (y), 3i+2 (z), the
// layout of libmorton's BMI2 masks (inc/encoding/libmorton/morton_BMI.h:40-58).
// Spread 21 bits to every third position with shift-and-mask steps.
__device__ __forceinline__ uint64_t spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}
__device__ __forceinline__ uint32_t compact3(uint64_t v) {
    v &= 0x1249249249249249ull;
    v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
    v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
    v = (v ^ (v >> 8)) & 0x1f0000ff0000ffull;
    v = (v ^ (v >> 16)) & 0x1f00000000ffffull;
    v = (v ^ (v >> 32)) & 0x1fffffull;
    return (uint32_t)v;
}
__device__ __forceinline__ uint64_t morton_encode(uint32_t x, uint32_t y, uint32_t z) {
    return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}
__device__ __forceinline__ void morton_decode(uint64_t k, uint32_t& x, uint32_t& y, uint32_t& z) {
    // the reference's X mask also covers key bit 63 (as coordinate bit 21)
    x = compact3(k) | (uint32_t)((k >> 63) << 21);
    y = compact3(k >> 1);
    z = compact3(k >> 2);
}

// Hilbert: HilbertEncoder3D::encode (inc/encoding/hilbert_encoder_3d.hpp:29-66),
// 21 levels from the top; the octant goes through {0,1,3,2,7,6,4,5}, then the
// coordinates are reflected and rotated (zi) or x/z swapped (!yi).
__device__ __forceinline__ uint64_t hilbert_encode(uint32_t x, uint32_t y, uint32_t z) {
    uint64_t key = 0;
#pragma unroll
    for (int level = (int)kMaxDepth - 1; level >= 0; --level) {
        const uint32_t xi = (x >> level) & 1u, yi = (y >> level) & 1u, zi = (z >> level) & 1u;
        const uint32_t oct = (xi << 2) | (yi << 1) | zi;
        // {0,1,3,2,7,6,4,5} packed as 3-bit fields
        const uint32_t digit = (0xB374C8u >> (3u * oct)) & 7u;
        key = (key << 3) | digit;
        const uint32_t nyi = yi ^ 1u, nzi = zi ^ 1u;
        x ^= 0u - (xi & (nyi | zi));
        y ^= 0u - ((xi & (yi | zi)) | (yi & nzi));
        z ^= 0u - ((xi & nyi & nzi) | (yi & nzi));
        if (zi) {
            const uint32_t t = x; x = y; y = z; z = t;
        } else if (!yi) {
            const uint32_t t = x; x = z; z = t;
        }
    }
    return key;
}

// HilbertEncoder3D::decode (hilbert_encoder_3d.hpp:256-289), from the lowest level.
__device__ __forceinline__ void hilbert_decode(uint64_t code, uint32_t& ox, uint32_t& oy, uint32_t& oz) {
    uint32_t x = 0, y = 0, z = 0;
#pragma unroll
    for (uint32_t level = 0; level < kMaxDepth; ++level) {
        const uint32_t oct = (uint32_t)(code >> (3 * level)) & 7u;
        const uint32_t xi = oct >> 2, yi = (oct >> 1) & 1u, zi = oct & 1u;
        if (yi ^ zi) {
            const uint32_t t = x; x = z; z = y; y = t;
        } else if (oct == 0u || oct == 7u) {
            const uint32_t t = x; x = z; z = t;
        }
        const uint32_t mask = (1u << level) - 1u;
        const uint32_t nxi = xi ^ 1u, nyi = yi ^ 1u, nzi = zi ^ 1u;
        x ^= mask & (0u - (xi & (yi | zi)));
        y ^= mask & (0u - ((xi & (nyi | nzi)) | (nxi & yi & zi)));
        z ^= mask & (0u - ((xi & nyi & nzi) | (yi & zi)));
        x |= xi << level;
        y |= (xi ^ yi) << level;
        z |= (yi ^ zi) << level;
    }
    ox = x; oy = y; oz = z;
}

// The same Hilbert keys from a 24-state automaton (states: the axis
// permutation and inversions the per-level transform has accumulated), as
// generated by csrc/gen_hilbert_table.py: entry = next_state << 3 | digit,
// indexed [state * 8 + octant of the ORIGINAL coordinates].  Kernels copy it
// to shared memory and pass it here.
constexpr int kHilbertStates = 24;
__device__ const uint8_t kHilbertTable[kHilbertStates * 8] = {
    160,  97,  11,  98, 183, 118,  12, 117,
    122,   3, 121, 184, 109,   4, 110, 175,
    126, 167, 125,  28, 105, 176, 106,  27,
     20, 101, 191, 102,  19, 114, 168, 113,
     96,  43, 161, 162, 119,  44, 182, 181,
    186, 185,  35, 120, 173, 174,  36, 111,
    190, 189, 103,  60, 169, 170, 112,  59,
     52, 127, 165, 166,  51, 104, 178, 177,
    128,  33, 151,  54,  75,  34,  76,  53,
     58,  67,  45,  68,  57, 152,  46, 143,
     62, 135,  41, 144,  61,  92,  42,  91,
     84,  37,  83,  50, 159,  38, 136,  49,
     32, 107,  55, 108, 129, 130, 150, 149,
    154, 153, 141, 142,  99,  56, 100,  47,
    158, 157, 137, 138,  39, 124,  48, 123,
    116,  63, 115,  40, 133, 134, 146, 145,
     64,  87,   1,  22, 139, 140,   2,  21,
     26,  13, 131, 132,  25,  14,  88,  79,
     30,   9,  71,  80,  29,  10, 156, 155,
    148, 147,   5,  18,  95,  72,   6,  17,
      0,  23, 171, 172,  65,  86,  66,  85,
     90,  77,  89,  78, 163, 164,  24,  15,
     94,  73,  93,  74,   7,  16, 188, 187,
    180, 179,  31,   8,  69,  82,  70,  81
};

__device__ __forceinline__ uint64_t hilbert_encode_tbl(uint32_t x, uint32_t y, uint32_t z, const uint8_t* tbl) {
    uint64_t key = 0;
    uint32_t st = 0;
#pragma unroll
    for (int level = (int)kMaxDepth - 1; level >= 0; --level) {
        const uint32_t o = (((x >> level) & 1u) << 2) | (((y >> level) & 1u) << 1) | ((z >> level) & 1u);
        const uint32_t e = tbl[st * 8 + o];
        key = (key << 3) | (e & 7u);
        st = e >> 3;
    }
    return key;
}

// Two levels per lookup: entry = next_state << 6 | first digit << 3 | second
// digit, indexed [state * 64 + octant at level L * 8 + octant at level L - 1],
// composed from kHilbertTable (the same walk, half the lookups).  The octant
// pairs come from one bit interleave with x in the high bit of each triple.
constexpr int kHilbertTable2Size = kHilbertStates * 64;
__device__ __forceinline__ void hilbert_table2_fill(uint16_t* t2, int tid, int nthreads) {
    for (int i = tid; i < kHilbertTable2Size; i += nthreads) {
        const uint32_t e1 = kHilbertTable[(i >> 6) * 8 + ((i >> 3) & 7)];
        const uint32_t e2 = kHilbertTable[(e1 >> 3) * 8 + (i & 7)];
        t2[i] = (uint16_t)(((e2 >> 3) << 6) | ((e1 & 7u) << 3) | (e2 & 7u));
    }
}
__device__ __forceinline__ uint64_t hilbert_encode_tbl2(uint32_t x, uint32_t y, uint32_t z, const uint8_t* t1,
                                                        const uint16_t* t2) {
    const uint64_t m = spread3(z) | (spread3(y) << 1) | (spread3(x) << 2);
    const uint32_t e = t1[(uint32_t)(m >> 60) & 7u];  // level 20 alone (21 levels)
    uint64_t key = e & 7u;
    uint32_t st = e >> 3;
#pragma unroll
    for (int level = 19; level > 0; level -= 2) {
        const uint32_t e2 = t2[st * 64 + ((uint32_t)(m >> (3 * (level - 1))) & 63u)];
        key = (key << 6) | (e2 & 63u);
        st = e2 >> 6;
    }
    return key;
}

// Anchor coordinate through a reciprocal: t' = x * RN(1 / 2r) differs from the
// reference's t = RN(x / 2r) by at most 1.5 * 2^-52 |t|, so for |t| <= 1 the
// scaled values differ by at most 2^-30.  When t' * 2^21 lies in [0, 2^21) and
// more than 2^-20 away from an integer, both truncate to the same coordinate;
// otherwise (boundaries, points outside the box, flat axes) the exact division
// decides.
__device__ __forceinline__ uint32_t anchor_coord_fast(double p, double c, double r, double inv2r) {
    const double x = dadd(dsub(p, c), r);
    const double v = dmul(dmul(x, inv2r), 2097152.0);
    if (v >= 0.0 && v < 2097152.0) {
        const double fl = floor(v);
        const double fr = dsub(v, fl);
        if (fr > 9.5367431640625e-07 && fr < 0.99999904632568359375) return (uint32_t)fl;
    }
    const double t = ddiv(x, dmul(2.0, r));
    const uint64_t u = x86_cvt_u64(dmul(t, 2097152.0));
    return (uint32_t)(u < kMaxCoord ? u : kMaxCoord);
}

template <int ENC>
__device__ __forceinline__ uint64_t sfc_encode(uint32_t x, uint32_t y, uint32_t z) {
    if constexpr (ENC == 5) return hilbert_encode(x, y, z);
    else return morton_encode(x, y, z);
}
template <int ENC>
__device__ __forceinline__ void sfc_decode(uint64_t k, uint32_t& x, uint32_t& y, uint32_t& z) {
    if constexpr (ENC == 5) hilbert_decode(k, x, y, z);
    else morton_decode(k, x, y, z);
}

// Key range of one node at `level` (PointEncoder::nodeRange, point_encoder.hpp:591-597).
__device__ __forceinline__ uint64_t node_range(uint32_t level) { return 1ull << (3u * (kMaxDepth - level)); }

// Node centre (PointEncoder::getCenter, point_encoder.hpp:517-539):
// decode the start key, mask the coordinates to the level, then
// min + c * half * 2 + radii[level] per axis.
template <int ENC>
__device__ __forceinline__ void node_center(uint64_t start_key, uint32_t level, const BoxD& box, const LevelGeom& g,
                                            double out[3]) {
    uint32_t c[3];
    sfc_decode<ENC>(start_key, c[0], c[1], c[2]);
    const uint32_t mask = ((1u << kMaxDepth) - 1u) ^ ((1u << (kMaxDepth - level)) - 1u);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double lo = dadd(box.min[a], dmul(dmul((double)(c[a] & mask), g.half[a]), 2.0));
        out[a] = dadd(lo, g.radii[level][a]);
    }
}

}  // namespace octb
