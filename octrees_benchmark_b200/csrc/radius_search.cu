// Fixed-radius search over the linear octree: neighbors, neighborsPrune and
// neighborsStruct with the sphere / cube / square / circle kernels.
//
// Reference path replaced: LinearOctree::singleTraversal (inc/structures/
// linear_octree.hpp:653-686) with the continuation criteria and leaf actions of
// neighborsStruct (695-736), neighborsPrune (746-784) and neighbors (796-816).
//
// B200 design: a group of G lanes (G = 8, 16 or 32; several queries per warp
// when G < 32) walks the tree for one query.  The group expands a node by
// judging its 8 children on 8 lanes at once (the reference's predicate, bit for
// bit), pushes the accepted children on a per-group shared-memory stack so that
// the lowest octant pops first, and scans leaves G points per step with a
// ballot to compact the hits.  Visiting octants in SFC order makes every
// query's output ascending.  A count pass sizes each query's output, a scan
// makes the CSR offsets, and a fill pass writes the indices (or ranges).
#include "cloud.h"
#include "search_kernels.cuh"

namespace octb {

namespace {

constexpr int kRadThreads = 256;
constexpr int kStackCap = 8 * (kMaxDepth + 1);  // 176 >= 7 * 21 + 8
enum : uint32_t { kKindExpand = 0, kKindScan = 1, kKindEmit = 2 };

struct RadiusArgs {
    const double* xs;
    const double* ys;
    const double* zs;
    const uint32_t* offsets;
    const uint2* ranges;
    const double* centers;
    const LevelGeom* geom;
    const double* q;        // nq x 3
    const double* qr;       // nq radii or nullptr
    double radius;
    uint64_t nq;
    unsigned long long* counts;        // count pass: results (indices, or ranges for struct)
    unsigned long long* counts2;       // count pass, struct: points
    const unsigned long long* offs;    // fill pass: CSR offsets
    uint32_t* out;                     // fill pass: indices, or (first, last) pairs for struct
    uint64_t out_cap;                  // entries (indices or pairs)
    uint32_t* err;
    uint32_t approx_cut;               // neighborsStruct: 0, or neighborsApprox's precisionLevel + 1
    uint32_t approx_upper;             // neighborsApprox: 1 adds the ranges of the cut octants
    const double* axes;                // per-axis radii (cube / square), or nullptr
    uint32_t axes_stride;              // 3: one (x, y, z) per query; 0: one for all queries
};

template <int G>
__device__ __forceinline__ uint32_t group_mask(int lane) {
    if constexpr (G == 32) return 0xffffffffu;
    else return ((1u << G) - 1u) << (lane & ~(G - 1));
}

template <int KT, int ALGO, int G, bool FILL>
__global__ void __launch_bounds__(kRadThreads) k_radius(RadiusArgs a) {
    constexpr int kGroups = kRadThreads / G;
    __shared__ uint32_t st_node[kGroups][kStackCap];
    __shared__ uint8_t st_meta[kGroups][kStackCap];
    __shared__ double s_radii[kMaxDepth + 1][3];

    for (int i = threadIdx.x; i < (kMaxDepth + 1) * 3; i += kRadThreads)
        (&s_radii[0][0])[i] = (&a.geom->radii[0][0])[i];
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int glane = lane & (G - 1);
    const int gib = threadIdx.x / G;  // group in block
    const uint32_t gmask = group_mask<G>(lane);
    const int gshift = lane & ~(G - 1);
    uint32_t* sn = st_node[gib];
    uint8_t* sm = st_meta[gib];

    const uint64_t ngroups = (uint64_t)gridDim.x * kGroups;
    for (uint64_t q = (uint64_t)blockIdx.x * kGroups + gib; q < a.nq; q += ngroups) {
        SearchKernel k;
        if (a.axes) k.init_axes(a.q[3 * q], a.q[3 * q + 1], a.q[3 * q + 2], a.axes + (uint64_t)a.axes_stride * q);
        else k.init(a.q[3 * q], a.q[3 * q + 1], a.q[3 * q + 2], a.qr ? a.qr[q] : a.radius);
        unsigned long long cnt = 0;   // indices (prune/neighbors) or ranges (struct)
        unsigned long long cnt2 = 0;  // struct: points
        unsigned long long base = 0;
        if (FILL) base = a.offs[q];
        bool overflow = false;

        // --- emit helpers (all lanes of the group call them uniformly) ---
        auto emit_range = [&](uint32_t f, uint32_t l) {
            if constexpr (ALGO == kStruct) {
                if (FILL && glane == 0) {
                    const unsigned long long o = base + cnt;
                    if (o < a.out_cap) {
                        a.out[2 * o] = f;
                        a.out[2 * o + 1] = l;
                    } else {
                        overflow = true;
                    }
                }
                cnt += 1;
                cnt2 += (unsigned long long)(l - f);
            } else {
                if (FILL) {
                    for (uint32_t i = f + glane; i < l; i += G) {
                        const unsigned long long o = base + cnt + (i - f);
                        if (o < a.out_cap) a.out[o] = i;
                        else overflow = true;
                    }
                }
                cnt += (unsigned long long)(l - f);
            }
        };
        auto scan_leaf = [&](uint32_t node) {
            const uint2 rg = a.ranges[node];
            if constexpr (ALGO == kStruct) {
                bool open = false;
                uint32_t rs = 0;
                for (uint32_t b = rg.x; b < rg.y; b += G) {
                    const uint32_t i = b + glane;
                    bool in = false;
                    if (i < rg.y) in = is_inside<KT>(k, a.xs[i], a.ys[i], a.zs[i]);
                    const uint32_t nvalid = (rg.y - b < (uint32_t)G) ? (rg.y - b) : (uint32_t)G;
                    const uint32_t vmask = (nvalid >= 32) ? 0xffffffffu : ((1u << nvalid) - 1u);
                    const uint32_t m = (__ballot_sync(gmask, in) >> gshift) & vmask;
                    uint32_t pos = 0;
                    while (pos < nvalid) {
                        const uint32_t from = (pos >= 32) ? 0u : (0xffffffffu << pos);
                        if (open) {
                            const uint32_t zeros = ~m & vmask & from;
                            if (!zeros) {
                                pos = nvalid;
                            } else {
                                const uint32_t e = __ffs(zeros) - 1;
                                emit_range(rs, b + e);
                                open = false;
                                pos = e + 1;
                            }
                        } else {
                            const uint32_t ones = m & from;
                            if (!ones) {
                                pos = nvalid;
                            } else {
                                const uint32_t s = __ffs(ones) - 1;
                                rs = b + s;
                                open = true;
                                pos = s + 1;
                            }
                        }
                    }
                }
                if (open) emit_range(rs, rg.y);
            } else {
                for (uint32_t b = rg.x; b < rg.y; b += G) {
                    const uint32_t i = b + glane;
                    bool in = false;
                    if (i < rg.y) in = is_inside<KT>(k, a.xs[i], a.ys[i], a.zs[i]);
                    const uint32_t m = __ballot_sync(gmask, in) >> gshift;
                    if (FILL && in) {
                        const unsigned long long o = base + cnt + __popc(m & ((1u << glane) - 1u));
                        if (o < a.out_cap) a.out[o] = i;
                        else overflow = true;
                    }
                    cnt += __popc(m);
                }
            }
        };

        // --- root: continuationCriterion(0, 0) ---
        int sp = 0;
        {
            const double* oc = a.centers;
            bool accept;
            bool inside = false;
            if constexpr (ALGO == kNeighbors) {
                accept = box_overlap<KT>(k, oc, s_radii[0]);
            } else {
                const int j = box_intersect<KT>(k, oc, s_radii[0]);
                inside = (j == kInside);
                accept = (j == kOverlap);
            }
            if (inside) {
                const uint2 rg = a.ranges[0];
                emit_range(rg.x, rg.y);
            } else if (accept) {
                if (a.offsets[0] == 0) scan_leaf(0);
                else {
                    if (glane == 0) { sn[0] = 0; sm[0] = (uint8_t)(kKindExpand << 5); }
                    sp = 1;
                }
            }
        }
        __syncwarp(gmask);
        while (sp > 0) {
            --sp;
            const uint32_t node = sn[sp];
            const uint32_t meta = sm[sp];
            __syncwarp(gmask);
            const uint32_t kind = meta >> 5, depth = meta & 31u;
            if (kind == kKindEmit) {
                const uint2 rg = a.ranges[node];
                emit_range(rg.x, rg.y);
            } else if (kind == kKindScan) {
                scan_leaf(node);
            } else {
                const uint32_t first_child = a.offsets[node];
                const uint32_t cd = depth + 1;
                uint32_t ckind = 0;
                bool push = false;
                if (glane < 8) {
                    const uint32_t child = first_child + glane;
                    const double* oc = a.centers + 3ull * child;
                    const bool leaf = a.offsets[child] == 0;
                    if constexpr (ALGO == kNeighbors) {
                        push = box_overlap<KT>(k, oc, s_radii[cd]);
                        ckind = leaf ? kKindScan : kKindExpand;
                    } else if (ALGO == kStruct && a.approx_cut != 0 && cd >= a.approx_cut) {
                        // neighborsApprox (linear_octree.hpp:979-985): below its precision level a
                        // child is cut before any box test, its whole range added in upper-bound mode
                        push = a.approx_upper != 0;
                        ckind = kKindEmit;
                    } else {
                        const int j = box_intersect<KT>(k, oc, s_radii[cd]);
                        push = (j != kOutside);
                        ckind = (j == kInside) ? kKindEmit : (leaf ? kKindScan : kKindExpand);
                    }
                }
                const uint32_t pm = (__ballot_sync(gmask, push) >> gshift) & 0xffu;
                const int npush = __popc(pm);
                if (sp + npush > kStackCap) {
                    overflow = true;
                    break;
                }
                if (push) {
                    // lowest octant on top of the stack
                    const int slot = sp + __popc(pm >> (glane + 1));
                    sn[slot] = first_child + glane;
                    sm[slot] = (uint8_t)((ckind << 5) | cd);
                }
                __syncwarp(gmask);
                sp += npush;
            }
        }
        if (overflow) set_err(a.err, FILL ? kErrOutputCapacity : kErrStackOverflow);
        if (!FILL && glane == 0) {
            a.counts[q] = cnt;
            if (ALGO == kStruct) a.counts2[q] = cnt2;
        }
        __syncwarp(gmask);
    }
}

// ---- exclusive scan of u64 counts into CSR offsets (n + 1 entries) ----
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ unsigned long long block_excl_scan(unsigned long long v, unsigned long long* red,
                                                              unsigned long long* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) red[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0ull;
        unsigned long long s = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, s, off);
            if (lane >= off) s += y;
        }
        if (lane < (int)(blockDim.x >> 5)) red[lane] = s - w;
        if (lane == 31) red[32] = s;
    }
    __syncthreads();
    const unsigned long long r = red[warp] + x - v;
    *total = red[32];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_partials(const unsigned long long* in, uint64_t n,
                                                                unsigned long long* partials) {
    __shared__ unsigned long long red[33];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    unsigned long long s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const uint64_t i = base + (uint64_t)threadIdx.x * kScanItems + j;
        if (i < n) s += in[i];
    }
    unsigned long long tot;
    block_excl_scan(s, red, &tot);
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_top(unsigned long long* partials, uint64_t m) {
    __shared__ unsigned long long red[33];
    unsigned long long carry = 0;
    for (uint64_t b = 0; b < m; b += kScanThreads) {
        const uint64_t i = b + threadIdx.x;
        const unsigned long long v = (i < m) ? partials[i] : 0ull;
        unsigned long long tot;
        const unsigned long long e = block_excl_scan(v, red, &tot);
        if (i < m) partials[i] = carry + e;
        carry += tot;
    }
    if (threadIdx.x == 0) partials[m] = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const unsigned long long* in, uint64_t n,
                                                             const unsigned long long* partials,
                                                             unsigned long long* out) {
    __shared__ unsigned long long red[33];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    unsigned long long v[kScanItems];
    unsigned long long s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const uint64_t i = base + (uint64_t)threadIdx.x * kScanItems + j;
        v[j] = (i < n) ? in[i] : 0ull;
        s += v[j];
    }
    unsigned long long tot;
    unsigned long long e = block_excl_scan(s, red, &tot) + partials[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        const uint64_t i = base + (uint64_t)threadIdx.x * kScanItems + j;
        if (i < n) out[i] = e;
        e += v[j];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = partials[gridDim.x];
}

int sm_count_r(int device) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v;
}

template <int KT, int ALGO, int G>
cudaError_t launch_one(const RadiusArgs& a, bool fill, int grid, cudaStream_t s) {
    if (fill) k_radius<KT, ALGO, G, true><<<grid, kRadThreads, 0, s>>>(a);
    else k_radius<KT, ALGO, G, false><<<grid, kRadThreads, 0, s>>>(a);
    return cudaGetLastError();
}

template <int KT, int ALGO>
cudaError_t launch_g(const RadiusArgs& a, int group, bool fill, int grid, cudaStream_t s) {
    switch (group) {
        case 8: return launch_one<KT, ALGO, 8>(a, fill, grid, s);
        case 16: return launch_one<KT, ALGO, 16>(a, fill, grid, s);
        default: return launch_one<KT, ALGO, 32>(a, fill, grid, s);
    }
}

template <int KT>
cudaError_t launch_a(const RadiusArgs& a, int algo, int group, bool fill, int grid, cudaStream_t s) {
    switch (algo) {
        case kNeighbors: return launch_g<KT, kNeighbors>(a, group, fill, grid, s);
        case kStruct: return launch_g<KT, kStruct>(a, group, fill, grid, s);
        default: return launch_g<KT, kPrune>(a, group, fill, grid, s);
    }
}

}  // namespace

cudaError_t launch_radius(Cloud& c, int kernel, int algo, int group, bool fill, const double* d_centers,
                          uint64_t nq, const double* d_radii, double radius, unsigned long long* d_counts,
                          unsigned long long* d_counts2, const unsigned long long* d_offsets, uint32_t* d_out,
                          uint64_t out_capacity) {
    if (nq == 0) return cudaSuccess;
    RadiusArgs a;
    a.xs = c.xs.as<double>();
    a.ys = c.ys.as<double>();
    a.zs = c.zs.as<double>();
    a.offsets = c.offsets.as<uint32_t>();
    a.ranges = c.ranges.as<uint2>();
    a.centers = c.centers.as<double>();
    a.geom = reinterpret_cast<const LevelGeom*>(c.d_box.as<unsigned char>() + sizeof(BoxD));
    a.q = d_centers;
    a.qr = d_radii;
    a.radius = radius;
    a.nq = nq;
    a.counts = d_counts;
    a.counts2 = d_counts2;
    a.offs = d_offsets;
    a.out = d_out;
    a.out_cap = out_capacity;
    a.err = c.d_err.as<uint32_t>();
    a.approx_cut = c.approx_cut;
    a.approx_upper = (uint32_t)c.approx_upper;
    a.axes = c.axes;
    a.axes_stride = c.axes_stride;
    const int groups_per_block = kRadThreads / group;
    const uint64_t want = (nq + groups_per_block - 1) / groups_per_block;
    const uint64_t cap = (uint64_t)sm_count_r(c.device) * 8;
    const int grid = (int)(want < cap ? want : cap);
    switch (kernel) {
        case kCircle: return launch_a<kCircle>(a, algo, group, fill, grid, c.stream);
        case kSquare: return launch_a<kSquare>(a, algo, group, fill, grid, c.stream);
        case kCube: return launch_a<kCube>(a, algo, group, fill, grid, c.stream);
        default: return launch_a<kSphere>(a, algo, group, fill, grid, c.stream);
    }
}

cudaError_t launch_scan_u64(Cloud& c, const unsigned long long* d_in, unsigned long long* d_out, uint64_t n) {
    cudaError_t e;
    const uint64_t blocks = (n + kScanTile - 1) / kScanTile;
    if ((e = c.q_scan_tmp.reserve(8 * (blocks + 2))) != cudaSuccess) return e;
    unsigned long long* part = c.q_scan_tmp.as<unsigned long long>();
    if (n == 0) return cudaMemsetAsync(d_out, 0, 8, c.stream);
    k_scan_partials<<<(unsigned)blocks, kScanThreads, 0, c.stream>>>(d_in, n, part);
    k_scan_top<<<1, kScanThreads, 0, c.stream>>>(part, blocks);
    k_scan_apply<<<(unsigned)blocks, kScanThreads, 0, c.stream>>>(d_in, n, part, d_out);
    return cudaGetLastError();
}

// A kernel of this file's device code, for preload_kernels.
const void* kernel_anchor_radius_search() { return reinterpret_cast<const void*>(&k_scan_top); }

}  // namespace octb
