// Linear-octree build over the SFC-sorted keys.
//
// Reference path replaced: LinearOctree::buildOctree (inc/structures/linear_octree.hpp:
// 567-605): the cornerstone leaf iteration (buildOctreeLeaves 458-471 with
// rebalanceDecision / calculateNodeOp / processNode / computeNodeCounts), then
// createUnsortedLayout, a sort of the Warren-Salmon prefixes, linkTree,
// computeInternalRanges and computeGeometry (336-565).
//
// Why a top-down construction gives the same arrays.  In the reference's
// iteration a leaf is split when its count exceeds maxPointsLeaf (and level <
// 21) and 8 sibling leaves merge when their summed count is <= maxPointsLeaf.
// Starting from the root, every split node had count > maxPointsLeaf, so its
// 8 children always sum above it and no merge ever fires: the converged tree
// is exactly "split every node with more than maxPointsLeaf points, down to
// level 21".  Sorting the nodes by their placeholder-bit prefix (1 followed by
// the 3*level key bits) orders them level by level and, inside a level, by key:
// breadth-first order.  So the node of child c of the j-th internal node of
// level l sits at level_start[l+1] + 8 j + c, and offsets[] of the k-th
// internal node of level l+1 is level_start[l+2] + 8 k.  internalRanges of a
// node are the lower_bounds of its start and end key in the sorted keys, and
// its centre is PointEncoder::getCenter of its start key.
//
// Kernel: one cooperative, persistent launch.  Per level, phase A computes the
// 8 children of every internal node (one lane per child: a binary search in the
// parent's point range, the centre, the split flag) and ballots the split flags
// per 32 children; phase B ranks the split children and writes the next
// frontier and the offsets.  A block's phase B reads only what its own phase A
// wrote, plus the number of split children of the blocks before it, which it
// takes by decoupled look-back over per-block status words (flag | count) —
// so one grid barrier per level (the next level reads every block's frontier)
// instead of two.  Grid barriers and look-back waits are bounded.
#include "cloud.h"
#include "sfc.cuh"

namespace octb {

namespace {

constexpr int kBuildThreads = 1024;
constexpr int kBuildWarps = kBuildThreads / 32;

struct FrontierNode {
    unsigned long long key;  // start key of the node
    uint32_t first, last;    // point range
};

struct BoxGeom {
    BoxD box;
    LevelGeom geom;
};

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// look-back status word of a block at one level: flag (bits 62-63) | split children (low 32 bits)
constexpr unsigned long long kLbLocal = 1ull << 62;   // this block's count
constexpr unsigned long long kLbPrefix = 2ull << 62;  // this block's and every earlier block's
constexpr unsigned long long kLbFlags = 3ull << 62;

// Grid-wide barrier for a cooperative launch; gives up after kSpinLimit polls.
__device__ void grid_barrier(BuildCtl* ctl, uint32_t* err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t gen = ld_acquire_u32(&ctl->barrier_gen);
        __threadfence();
        const uint32_t arrived = atomicAdd(&ctl->barrier_count, 1u) + 1u;
        if (arrived == gridDim.x) {
            atomicExch(&ctl->barrier_count, 0u);
            __threadfence();
            atomicAdd(&ctl->barrier_gen, 1u);
        } else {
            uint32_t spins = 0;
            while (ld_acquire_u32(&ctl->barrier_gen) == gen) {
                if (++spins > kSpinLimit) {
                    set_err(err, kErrSpinLimit);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// lower_bound over a child's parent range.  Ranges longer than kKaryMin are
// first narrowed kKaryWays-fold per step by kKaryWays - 1 independent probes
// (one round trip each step instead of log2(kKaryWays) dependent ones: the top
// levels' searches span millions of keys), then bisected.
constexpr uint32_t kKaryWays = 8;
constexpr uint32_t kKaryMin = 256;
static_assert(kKaryMin >= kKaryWays, "a k-ary step needs a stride of at least one key");

__device__ __forceinline__ uint32_t lower_bound_keys(const uint64_t* __restrict__ keys, uint32_t lo, uint32_t hi,
                                                     uint64_t v) {
    while (hi - lo > kKaryMin) {
        // keys [lo, hi) ascending; the answer lies in [lo, hi]
        const uint32_t s = (hi - lo) / kKaryWays;
        uint32_t below = 0;  // probes lo + p s (p = 1 .. ways - 1) under v: a prefix of them
#pragma unroll
        for (uint32_t p = 1; p < kKaryWays; ++p) below += keys[lo + p * s] < v ? 1u : 0u;
        const uint32_t nlo = below ? lo + below * s + 1 : lo;
        if (below < kKaryWays - 1) hi = lo + (below + 1) * s;
        lo = nlo;
    }
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (keys[mid] < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Block-wide sum of one value per thread.
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* red) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    uint32_t s = 0;
    for (int w = 0; w < kBuildWarps; ++w) s += red[w];
    return s;
}

template <int ENC>
__global__ void __launch_bounds__(kBuildThreads) k_build(const uint64_t* __restrict__ keys, uint32_t n,
                                                         uint32_t max_leaf, const BoxGeom* __restrict__ bgp,
                                                         uint32_t* __restrict__ offsets, uint2* __restrict__ ranges,
                                                         double* __restrict__ centers, uint32_t node_cap,
                                                         FrontierNode* __restrict__ fa, FrontierNode* __restrict__ fb,
                                                         uint32_t* __restrict__ masks,
                                                         unsigned long long* __restrict__ lb, BuildCtl* ctl,
                                                         uint32_t* err) {
    __shared__ BoxGeom bg;
    __shared__ uint32_t red[kBuildWarps];
    __shared__ uint32_t chunk_pre[kBuildThreads];
    __shared__ uint32_t s_excl;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) bg = *bgp;
    __syncthreads();

    // root (level 0): one block writes it
    if (blockIdx.x == 0 && tid == 0) {
        double c[3];
        node_center<ENC>(0ull, 0, bg.box, bg.geom, c);
        centers[0] = c[0]; centers[1] = c[1]; centers[2] = c[2];
        ranges[0] = make_uint2(0u, n);
        const bool split = n > max_leaf;  // level 0 < 21
        offsets[0] = split ? 1u : 0u;
        ctl->level_start[0] = 0;
        ctl->level_start[1] = 1;
        ctl->level_internal[0] = split ? 1u : 0u;
        ctl->n_internal = split ? 1u : 0u;
        ctl->max_depth_seen = split ? 1u : 0u;
        ctl->n_total = 1;
        if (split) {
            FrontierNode r;
            r.key = 0ull; r.first = 0u; r.last = n;
            fa[0] = r;
        }
    }
    grid_barrier(ctl, err);

    FrontierNode* cur = fa;
    FrontierNode* nxt = fb;
    uint32_t F = ld_acquire_u32(&ctl->level_internal[0]);
    uint32_t n_internal = F;
    // first node of the level being created, kept by every block (block 0 writes the
    // level starts for the host after the level's barrier, so they are not read back here)
    uint32_t level_first = 1;
    for (uint32_t l = 0; l < kMaxDepth && F > 0; ++l) {
        const uint32_t child_level = l + 1;
        const uint32_t lstart = level_first;
        const uint64_t nchild = 8ull * F;
        const uint64_t next_start = (uint64_t)lstart + nchild;
        if (next_start > node_cap) {  // uniform across blocks: every block sees the same values
            if (blockIdx.x == 0 && tid == 0) {
                ctl->need_nodes = (uint32_t)(next_start < 0xffffffffull ? next_start : 0xffffffffull);
                set_err(err, kErrNodeCapacity);
            }
            break;
        }
        const uint64_t crange = node_range(child_level);
        const uint32_t W = (uint32_t)((nchild + 31) / 32);
        const uint32_t C = (W + gridDim.x - 1) / gridDim.x;
        const uint32_t w0 = blockIdx.x * C;
        const uint32_t w1 = (w0 + C < W) ? (w0 + C) : W;
        // ---- phase A: children, their ranges and centres, split ballots ----
        uint32_t my_count = 0;
        for (uint32_t w = w0 + warp; w < w1; w += kBuildWarps) {
            const uint64_t t = 32ull * w + lane;
            const bool valid = t < nchild;
            uint32_t first = 0, last = 0;
            bool split = false;
            if (valid) {
                const uint32_t j = (uint32_t)(t >> 3), c = (uint32_t)(t & 7);
                const FrontierNode p = cur[j];
                const uint64_t ck = p.key + (uint64_t)c * crange;
                first = (c == 0) ? p.first : lower_bound_keys(keys, p.first, p.last, ck);
                const uint32_t node = lstart + (uint32_t)t;
                double cc[3];
                node_center<ENC>(ck, child_level, bg.box, bg.geom, cc);
                centers[3ull * node] = cc[0];
                centers[3ull * node + 1] = cc[1];
                centers[3ull * node + 2] = cc[2];
                last = p.last;  // child 7; others take the next child's first below
            }
            const uint32_t nf = __shfl_down_sync(0xffffffffu, first, 1);
            if (valid) {
                const uint32_t c = (uint32_t)(t & 7);
                if (c != 7) last = nf;
                const uint32_t node = lstart + (uint32_t)t;
                ranges[node] = make_uint2(first, last);
                split = (last - first > max_leaf) && (child_level < kMaxDepth);
                offsets[node] = 0u;
            }
            const uint32_t m = __ballot_sync(0xffffffffu, split);
            if (lane == 0) {
                masks[w] = m;
                my_count += __popc(m);
            }
        }
        const uint32_t bsum = block_sum(my_count, red);
        // ---- the split children of the blocks before this one: decoupled look-back ----
        unsigned long long* st = lb + (uint64_t)l * gridDim.x;
        if (warp == 0) {
            if (lane == 0)
                st_release_u64(&st[blockIdx.x], (blockIdx.x == 0 ? kLbPrefix : kLbLocal) | bsum);
            uint32_t excl = 0;
            int64_t t = (int64_t)blockIdx.x - 1;  // the nearest predecessor not summed yet
            uint32_t spins = 0;
            while (t >= 0) {
                const int64_t ti = t - lane;  // lane 0: the nearest
                const unsigned long long v = ti >= 0 ? ld_acquire_u64(&st[ti]) : kLbPrefix;
                const uint32_t ready = __ballot_sync(0xffffffffu, (v & kLbFlags) != 0);
                const uint32_t pref = __ballot_sync(0xffffffffu, (v & kLbFlags) == kLbPrefix);
                // lanes up to the nearest prefix must all have published; else wait for them
                const uint32_t upto = pref ? ((pref & (0u - pref)) << 1) - 1u : 0xffffffffu;
                if ((ready & upto) != upto) {
                    if (++spins > kSpinLimit) {
                        if (lane == 0) set_err(err, kErrSpinLimit);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                uint32_t c = ((upto >> lane) & 1u) && ti >= 0 ? (uint32_t)(v & 0xffffffffull) : 0u;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
                excl += c;
                if (pref) break;
                t -= 32;
            }
            if (lane == 0) {
                if (blockIdx.x > 0) st_release_u64(&st[blockIdx.x], kLbPrefix | (excl + bsum));
                s_excl = excl;
            }
        }
        __syncthreads();
        // ---- phase B: rank split children, next frontier, offsets ----
        const uint32_t pre = s_excl;
        const uint32_t next_level_start = (uint32_t)next_start;
        uint32_t carry = pre;
        for (uint32_t seg = w0; seg < w1; seg += kBuildThreads) {
            const uint32_t i = seg + tid;
            const uint32_t v = (i < w1) ? __popc(((volatile uint32_t*)masks)[i]) : 0u;
            // block exclusive scan of v
            uint32_t x = v;
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
                if (lane >= off) x += y;
            }
            __syncthreads();
            if (lane == 31) red[warp] = x;
            __syncthreads();
            uint32_t wp = 0, segsum = 0;
            for (int ww = 0; ww < kBuildWarps; ++ww) {
                if (ww < warp) wp += red[ww];
                segsum += red[ww];
            }
            chunk_pre[tid] = carry + wp + x - v;
            __syncthreads();
            const uint32_t seg_end = (seg + kBuildThreads < w1) ? seg + kBuildThreads : w1;
            for (uint32_t w = seg + warp; w < seg_end; w += kBuildWarps) {
                const uint32_t m = ((volatile uint32_t*)masks)[w];
                if (m & (1u << lane)) {
                    const uint32_t rank = chunk_pre[w - seg] + __popc(m & lanemask_lt());
                    const uint64_t t = 32ull * w + lane;
                    const uint32_t node = lstart + (uint32_t)t;
                    const FrontierNode p = cur[t >> 3];
                    const uint2 rg = ranges[node];
                    FrontierNode q;
                    q.key = p.key + (t & 7) * crange;
                    q.first = rg.x;
                    q.last = rg.y;
                    nxt[rank] = q;
                    offsets[node] = next_level_start + 8u * rank;
                }
            }
            carry += segsum;
            __syncthreads();
        }
        grid_barrier(ctl, err);
        // every block has published its inclusive prefix before the barrier: the last one's is the total
        const uint32_t tot = (uint32_t)(ld_acquire_u64(&st[gridDim.x - 1]) & 0xffffffffull);
        if (blockIdx.x == 0 && tid == 0) {
            ctl->level_start[l + 2] = next_level_start;
            ctl->level_internal[l + 1] = tot;
            ctl->n_total = next_level_start;
            if (tot > 0) ctl->max_depth_seen = l + 2;
        }
        n_internal += tot;
        level_first = next_level_start;
        FrontierNode* tmp = cur;
        cur = nxt;
        nxt = tmp;
        F = tot;
    }
    if (blockIdx.x == 0 && tid == 0) ctl->n_internal = n_internal;
}

int sm_count_b(int device) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v;
}

}  // namespace

cudaError_t launch_build(Cloud& c, bool* capacity_ok) {
    cudaError_t e;
    *capacity_ok = true;
    const uint64_t n = c.n;
    const uint32_t M = c.params.max_points_leaf;
    if (c.node_capacity == 0) {
        // nodes = 1 + 8 * internal; a level holds at most n / (M + 1) internal nodes
        const uint64_t per_level = n / ((uint64_t)M + 1) + 1;
        uint64_t cap = 8 * 3 * per_level + 9;
        if (cap > 0xfffffff0ull) cap = 0xfffffff0ull;
        c.node_capacity = (uint32_t)cap;
    }
    const uint64_t cap = c.node_capacity;
    const uint64_t fcap = n / ((uint64_t)M + 1) + 2;
    if ((e = c.offsets.reserve(4 * (cap + 1))) != cudaSuccess) return e;
    if ((e = c.ranges.reserve(8 * cap)) != cudaSuccess) return e;
    if ((e = c.centers.reserve(24 * cap)) != cudaSuccess) return e;
    if ((e = c.frontier.reserve(2 * sizeof(FrontierNode) * fcap)) != cudaSuccess) return e;
    if ((e = c.masks.reserve(4 * ((8 * fcap + 31) / 32 + 1))) != cudaSuccess) return e;

    int dev = c.device;
    int per_sm = 0;
    void (*kfn)(const uint64_t*, uint32_t, uint32_t, const BoxGeom*, uint32_t*, uint2*, double*, uint32_t,
                FrontierNode*, FrontierNode*, uint32_t*, unsigned long long*, BuildCtl*, uint32_t*) =
        (c.params.encoder == OCT_ENC_HILBERT_3D) ? k_build<5> : k_build<1>;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kBuildThreads, 0)) != cudaSuccess)
        return e;
    if (per_sm < 1) per_sm = 1;
    if (per_sm > 4) per_sm = 4;
    unsigned grid = (unsigned)(sm_count_b(dev) * per_sm);
    // small trees need few blocks; keep at least one
    const uint64_t max_useful = (8 * fcap + 31) / 32 / kBuildWarps + 1;
    if (grid > max_useful) grid = (unsigned)max_useful;
    if (grid < 1) grid = 1;
    // BuildCtl, then the look-back status words of every level and block (zeroed: no flag)
    const size_t ctl_bytes = (sizeof(BuildCtl) + 255) / 256 * 256;
    const size_t lb_bytes = sizeof(unsigned long long) * (kMaxDepth + 1) * (size_t)grid;
    if ((e = c.d_build.reserve(ctl_bytes + lb_bytes)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(c.d_build.ptr, 0, ctl_bytes + lb_bytes, c.stream)) != cudaSuccess) return e;

    const uint64_t* keys = c.keys.as<uint64_t>();
    uint32_t nn = (uint32_t)n;
    uint32_t ml = M;
    const BoxGeom* bg = c.d_box.as<BoxGeom>();
    uint32_t* offs = c.offsets.as<uint32_t>();
    uint2* rng = c.ranges.as<uint2>();
    double* ctr = c.centers.as<double>();
    uint32_t ncap = (uint32_t)cap;
    FrontierNode* fa = c.frontier.as<FrontierNode>();
    FrontierNode* fb = fa + fcap;
    uint32_t* masks = c.masks.as<uint32_t>();
    BuildCtl* ctl = c.d_build.as<BuildCtl>();
    unsigned long long* lb = reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(c.d_build.ptr) +
                                                                   ctl_bytes);
    uint32_t* err = c.d_err.as<uint32_t>();
    void* args[] = {(void*)&keys, &nn, &ml, (void*)&bg, &offs, &rng, &ctr, &ncap, &fa, &fb, &masks, &lb,
                    &ctl, &err};
    e = cudaLaunchCooperativeKernel((const void*)kfn, dim3(grid), dim3(kBuildThreads), args, 0, c.stream);
    return e;
}

// A kernel of this file's device code, for preload_kernels.
const void* kernel_anchor_octree_build() { return reinterpret_cast<const void*>(&k_build<1>); }

}  // namespace octb
