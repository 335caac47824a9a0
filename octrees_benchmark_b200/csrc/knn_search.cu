// k nearest neighbours over the linear octree.
//
// Reference path replaced: LinearOctree::knn (inc/structures/linear_octree.hpp:
// 899-942), a best-first search over one heap of octants (keyed by the
// clamp-to-box distance, distPointOctantSquared 854-878) and points (keyed by
// distPointsSquared 844-851) that stops after min(n, k) points.
//
// B200 design: one warp per query walks the tree depth-first, nearest child
// first (children of a node are judged on 8 lanes and ordered by their
// lower bound), and prunes every octant whose lower bound exceeds the current
// k-th distance.  The k best (squared distance, index) pairs live in a sorted
// list in shared memory; leaf points that beat the k-th pair are appended to a
// candidate buffer with a ballot, and a full buffer is merged into the list by
// a bitonic sort.  All distances are the reference's FP64 expressions, so the
// returned squared distances are bitwise the reference's, and ordering by
// (distance, index) resolves ties at the k-th distance by the lowest index.
#include <cfloat>

#include "cloud.h"
#include "search_kernels.cuh"

namespace octb {

namespace {

constexpr int kKnnWarps = 4;
constexpr int kKnnThreads = 32 * kKnnWarps;
constexpr int kKnnStack = 8 * (kMaxDepth + 1);

struct KnnArgs {
    const double* xs;
    const double* ys;
    const double* zs;
    const uint32_t* offsets;
    const uint2* ranges;
    const double* centers;
    const LevelGeom* geom;
    const double* q;
    uint64_t nq;
    uint32_t k;
    uint32_t* idx;
    double* d2;
    uint32_t* counts;
    uint32_t* err;
};

__device__ __forceinline__ bool pair_less(double da, uint32_t ia, double db, uint32_t ib) {
    return (da < db) || (da == db && ia < ib);
}

// Bitonic sort of P (power of two) (dist, idx) pairs in shared memory, one warp.
template <int P>
__device__ __forceinline__ void warp_bitonic_sort(double* d, uint32_t* ix) {
    const int lane = threadIdx.x & 31;
    for (int size = 2; size <= P; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = lane; i < P / 2; i += 32) {
                const int lo = 2 * stride * (i / stride) + (i % stride);
                const int hi = lo + stride;
                const bool asc = (lo & size) == 0;
                const double a = d[lo], b = d[hi];
                const uint32_t ia = ix[lo], ib = ix[hi];
                const bool swap = asc ? pair_less(b, ib, a, ia) : pair_less(a, ia, b, ib);
                if (swap) {
                    d[lo] = b; d[hi] = a;
                    ix[lo] = ib; ix[hi] = ia;
                }
            }
            __syncwarp();
        }
    }
}

// LCAP: list capacity (power of two >= k); the candidate buffer has LCAP slots too.
template <int LCAP>
__global__ void __launch_bounds__(kKnnThreads) k_knn(KnnArgs a) {
    constexpr int P = 2 * LCAP;
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // per warp: list+buffer (P pairs) and the traversal stack (node, depth, lower bound)
    double* base_d = reinterpret_cast<double*>(smem);
    double* sd = base_d + (size_t)warp * P;
    double* st_lb = base_d + (size_t)kKnnWarps * P + (size_t)warp * kKnnStack;
    uint32_t* base_u = reinterpret_cast<uint32_t*>(base_d + (size_t)kKnnWarps * (P + kKnnStack));
    uint32_t* si = base_u + (size_t)warp * P;
    uint32_t* st_node = base_u + (size_t)kKnnWarps * P + (size_t)warp * kKnnStack;
    uint8_t* st_depth =
        reinterpret_cast<uint8_t*>(base_u + (size_t)kKnnWarps * (P + kKnnStack)) + (size_t)warp * kKnnStack;
    __shared__ double s_radii[kMaxDepth + 1][3];
    for (int i = threadIdx.x; i < (kMaxDepth + 1) * 3; i += kKnnThreads) (&s_radii[0][0])[i] = (&a.geom->radii[0][0])[i];
    __syncthreads();

    const uint32_t K = a.k;
    const uint64_t nwarps = (uint64_t)gridDim.x * kKnnWarps;
    for (uint64_t q = (uint64_t)blockIdx.x * kKnnWarps + warp; q < a.nq; q += nwarps) {
        const double p[3] = {a.q[3 * q], a.q[3 * q + 1], a.q[3 * q + 2]};
        for (int i = lane; i < P; i += 32) {
            sd[i] = INFINITY;
            si[i] = 0xffffffffu;
        }
        __syncwarp();
        uint32_t nl = 0;        // entries in the sorted list sd[0, LCAP)
        uint32_t nb = 0;        // entries in the buffer sd[LCAP, 2 LCAP)
        double thr = INFINITY;  // k-th best distance (when nl == K)
        uint32_t thr_i = 0xffffffffu;
        bool failed = false;

        auto merge = [&]() {
            warp_bitonic_sort<P>(sd, si);
            uint32_t tot = nl + nb;
            nl = tot < K ? tot : K;
            nb = 0;
            for (int i = (int)nl + lane; i < P; i += 32) {
                sd[i] = INFINITY;
                si[i] = 0xffffffffu;
            }
            __syncwarp();
            if (nl == K) {
                thr = sd[K - 1];
                thr_i = si[K - 1];
            }
        };

        // stack of (node, depth, lower bound); the root's bound is 0 (linear_octree.hpp:904)
        if (lane == 0) {
            st_node[0] = 0;
            st_depth[0] = 0;
            st_lb[0] = 0.0;
        }
        __syncwarp();
        int sp = 1;
        while (sp > 0 && !failed) {
            --sp;
            const uint32_t node = st_node[sp];
            const double lb = st_lb[sp];
            const uint32_t depth = st_depth[sp];
            __syncwarp();
            if (lb > thr) continue;
            const uint32_t fc = a.offsets[node];
            if (fc == 0) {
                // leaf: distances of its points, candidates into the buffer
                const uint2 rg = a.ranges[node];
                for (uint32_t b = rg.x; b < rg.y; b += 32) {
                    const uint32_t i = b + lane;
                    double d = INFINITY;
                    bool cand = false;
                    if (i < rg.y) {
                        d = dist_pp(p[0], p[1], p[2], a.xs[i], a.ys[i], a.zs[i]);
                        cand = pair_less(d, i, thr, thr_i);
                    }
                    uint32_t m = __ballot_sync(0xffffffffu, cand);
                    if (nb + __popc(m) > (uint32_t)LCAP) {
                        merge();
                        cand = cand && pair_less(d, i, thr, thr_i);
                        m = __ballot_sync(0xffffffffu, cand);
                    }
                    if (cand) {
                        const uint32_t slot = LCAP + nb + __popc(m & lanemask_lt());
                        sd[slot] = d;
                        si[slot] = i;
                    }
                    nb += __popc(m);
                    __syncwarp();
                }
            } else {
                // internal: lower bounds of the 8 children, nearest pushed last
                const uint32_t cd = depth + 1;
                double clb = INFINITY;
                bool keep = false;
                if (lane < 8) {
                    clb = dist_po(p, a.centers + 3ull * (fc + lane), s_radii[cd]);
                    keep = !(clb > thr);
                }
                const uint32_t km = __ballot_sync(0xffffffffu, keep) & 0xffu;
                const int nk = __popc(km);
                if (sp + nk > kKnnStack) {
                    failed = true;
                    break;
                }
                // position among kept children by descending (lb, lane): farthest deepest
                int pos = 0;
#pragma unroll
                for (int o = 0; o < 8; ++o) {
                    const double ol = __shfl_sync(0xffffffffu, clb, o);
                    const bool ok = (km >> o) & 1u;
                    if (ok && o != lane && ((ol > clb) || (ol == clb && o > lane))) ++pos;
                }
                if (keep) {
                    const int slot = sp + pos;
                    st_node[slot] = fc + lane;
                    st_lb[slot] = clb;
                    st_depth[slot] = (uint8_t)cd;
                }
                __syncwarp();
                sp += nk;
            }
        }
        if (failed) set_err(a.err, kErrStackOverflow);
        if (nb > 0) merge();
        const uint64_t o = q * (uint64_t)K;
        for (uint32_t j = lane; j < K; j += 32) {
            if (j < nl) {
                a.idx[o + j] = si[j];
                a.d2[o + j] = sd[j];
            } else {
                a.idx[o + j] = 0xffffffffu;
                a.d2[o + j] = INFINITY;
            }
        }
        if (lane == 0 && a.counts) a.counts[q] = nl;
        __syncwarp();
    }
}

template <int LCAP>
size_t knn_smem() {
    const size_t P = 2 * LCAP;
    const size_t per = P + kKnnStack;
    return (size_t)kKnnWarps * (per * 8 + per * 4 + kKnnStack) + 16;
}

template <int LCAP>
cudaError_t launch_l(const KnnArgs& a, int grid, cudaStream_t s) {
    const size_t smem = knn_smem<LCAP>();
    cudaError_t e = cudaFuncSetAttribute(k_knn<LCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_knn<LCAP><<<grid, kKnnThreads, smem, s>>>(a);
    return cudaGetLastError();
}

int sm_count_k(int device) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v;
}

}  // namespace

cudaError_t launch_knn(Cloud& c, const double* d_centers, uint64_t nq, uint32_t k, uint32_t* d_idx, double* d_d2,
                       uint32_t* d_counts) {
    if (nq == 0 || k == 0) return cudaSuccess;
    KnnArgs a;
    a.xs = c.xs.as<double>();
    a.ys = c.ys.as<double>();
    a.zs = c.zs.as<double>();
    a.offsets = c.offsets.as<uint32_t>();
    a.ranges = c.ranges.as<uint2>();
    a.centers = c.centers.as<double>();
    a.geom = reinterpret_cast<const LevelGeom*>(c.d_box.as<unsigned char>() + sizeof(BoxD));
    a.q = d_centers;
    a.nq = nq;
    a.k = k;
    a.idx = d_idx;
    a.d2 = d_d2;
    a.counts = d_counts;
    a.err = c.d_err.as<uint32_t>();
    const uint64_t want = (nq + kKnnWarps - 1) / kKnnWarps;
    const uint64_t cap = (uint64_t)sm_count_k(c.device) * 16;
    const int grid = (int)(want < cap ? want : cap);
    if (k <= 32) return launch_l<32>(a, grid, c.stream);
    if (k <= 64) return launch_l<64>(a, grid, c.stream);
    if (k <= 128) return launch_l<128>(a, grid, c.stream);
    if (k <= 256) return launch_l<256>(a, grid, c.stream);
    if (k <= 512) return launch_l<512>(a, grid, c.stream);
    return launch_l<1024>(a, grid, c.stream);
}

}  // namespace octb
