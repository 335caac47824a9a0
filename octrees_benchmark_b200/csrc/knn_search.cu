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
// candidate buffer with a ballot, and a full buffer is sorted (descending) and
// bitonic-merged into the list.  All distances are the reference's FP64 expressions, so the
// returned squared distances are bitwise the reference's, and ordering by
// (distance, index) resolves ties at the k-th distance by the lowest index.
#include <algorithm>
#include <cfloat>
#include <cuda_fp16.h>

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
    const uint32_t* order;  // query visiting order (curve order), or nullptr
    uint32_t bucket;        // subtrees with at most this many points are scanned as one range
    const DynGroup* grp;    // table launch (k_knn<LCAP, true>): sizes and requests on the device
};

__device__ __forceinline__ bool pair_less(double da, uint32_t ia, double db, uint32_t ib) {
    return (da < db) || (da == db && ia < ib);
}

// Bitonic sort of N (power of two) pairs in shared memory into descending order, one warp.
template <int N>
__device__ __forceinline__ void warp_bitonic_sort_desc(double* d, uint32_t* ix) {
    const int lane = threadIdx.x & 31;
    for (int size = 2; size <= N; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = lane; i < N / 2; i += 32) {
                const int lo = ((i & ~(stride - 1)) << 1) | (i & (stride - 1));
                const int hi = lo + stride;
                const bool asc = (lo & size) != 0;  // mirrored network: the last stage runs descending
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

// A bitonic sequence of N (power of two) pairs into ascending order, one warp.
template <int N>
__device__ __forceinline__ void warp_bitonic_merge(double* d, uint32_t* ix) {
    const int lane = threadIdx.x & 31;
    for (int stride = N >> 1; stride > 0; stride >>= 1) {
        for (int i = lane; i < N / 2; i += 32) {
            const int lo = ((i & ~(stride - 1)) << 1) | (i & (stride - 1));
            const int hi = lo + stride;
            const double a = d[lo], b = d[hi];
            const uint32_t ia = ix[lo], ib = ix[hi];
            if (pair_less(b, ib, a, ia)) {
                d[lo] = b; d[hi] = a;
                ix[lo] = ib; ix[hi] = ia;
            }
        }
        __syncwarp();
    }
}

// LCAP: list capacity (power of two >= k); the candidate buffer has LCAP slots too.
// MULTI: a table launch (the batched engine): each query's request gives its
// cloud (kept per warp in shared memory), k and output slots.
// CARRY: children's records are read when their parent is expanded and carried
// on the stack (no dependent loads at a pop, empty leaves never pushed, subtrees
// of at most `bucket` points scanned as one range); without it (the plain path)
// a popped node's record is read then, one leaf at a time.
#define KV(f) (MULTI ? s_view[warp].f : a.f)
template <int LCAP, bool MULTI, bool CARRY = true>
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
    // stack entry: a range [st_a, st_b) to scan, or (st_b == 0xffffffff) an internal node whose first child is st_a
    uint32_t* st_a = base_u + (size_t)kKnnWarps * P + (size_t)warp * kKnnStack;
    uint32_t* st_b = base_u + (size_t)kKnnWarps * (P + kKnnStack) + (size_t)warp * kKnnStack;
    uint8_t* st_depth =
        reinterpret_cast<uint8_t*>(base_u + (size_t)kKnnWarps * (P + 2 * kKnnStack)) + (size_t)warp * kKnnStack;
    __shared__ double s_rad[MULTI ? kKnnWarps : 1][kMaxDepth + 1][3];
    __shared__ CloudView s_view[MULTI ? kKnnWarps : 1];
    double (*s_radii)[3] = s_rad[MULTI ? warp : 0];
    if (!MULTI) {
        for (int i = threadIdx.x; i < (kMaxDepth + 1) * 3; i += kKnnThreads)
            (&s_radii[0][0])[i] = (&a.geom->radii[0][0])[i];
        __syncthreads();
    }
    const SearchReq* reqs = nullptr;
    uint32_t nreq = 1, cur_cloud = 0xffffffffu;
    uint64_t q0 = 0, nq = a.nq;
    if (MULTI) {
        reqs = a.grp->reqs;
        nreq = a.grp->nreq;
        q0 = a.grp->q_begin;
        nq = a.grp->nq;
    }
    const uint64_t nwarps = (uint64_t)gridDim.x * kKnnWarps;
    for (uint64_t w = (uint64_t)blockIdx.x * kKnnWarps + warp; w < nq; w += nwarps) {
        const uint64_t qpos = q0 + w;
        const uint64_t q = a.order ? a.order[qpos] : qpos;
        uint32_t K = a.k;
        uint64_t o = q * (uint64_t)K;  // first output slot of this query
        const double* qc = a.q + 3 * q;
        if (MULTI) {  // the request whose positions contain qpos (q_begin ascending)
            uint32_t lo = 0, hi = nreq;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (reqs[mid].q_begin <= qpos) lo = mid;
                else hi = mid;
            }
            const SearchReq& rq = reqs[lo];
            if (rq.cloud_id != cur_cloud) {
                __syncwarp();
                const double* gr = &rq.cv.geom->radii[0][0];
                for (int t = lane; t < (kMaxDepth + 1) * 3; t += 32) (&s_radii[0][0])[t] = gr[t];
                if (lane == 0) s_view[warp] = rq.cv;
                cur_cloud = rq.cloud_id;
                __syncwarp();
            }
            K = rq.k;
            const uint64_t ql = q - rq.q_begin;
            o = rq.out_begin + ql * (uint64_t)K;
            qc = rq.centers + 3 * ql;
        }
        const double p[3] = {qc[0], qc[1], qc[2]};
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
            // the list half is sorted already: sort the buffer half descending, then one
            // bitonic merge of (ascending list, descending buffer) sorts all P pairs
            warp_bitonic_sort_desc<LCAP>(sd + LCAP, si + LCAP);
            warp_bitonic_merge<P>(sd, si);
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

        // stack of (range or first child, depth, lower bound); the root's bound is 0
        // (linear_octree.hpp:904).  Child records are read when their parent is
        // expanded, so a popped entry needs no further dependent loads; empty leaves
        // are never pushed and subtrees of at most `bucket` points are scanned as one
        // range (extra points cannot change the k best pairs).
        if constexpr (CARRY) {
            const uint32_t fc0 = KV(offsets)[0];
            const uint2 rg0 = KV(ranges)[0];
            const bool scan0 = fc0 == 0 || rg0.y - rg0.x <= a.bucket;
            if (lane == 0) {
                st_a[0] = scan0 ? rg0.x : fc0;
                st_b[0] = scan0 ? rg0.y : 0xffffffffu;
                st_depth[0] = 0;
                st_lb[0] = 0.0;
            }
        } else if (lane == 0) {
            st_a[0] = 0;  // the root node
            st_depth[0] = 0;
            st_lb[0] = 0.0;
        }
        __syncwarp();
        int sp = 1;
        while (sp > 0 && !failed) {
            --sp;
            uint32_t ea = st_a[sp], eb = st_b[sp];
            const double lb = st_lb[sp];
            const uint32_t depth = st_depth[sp];
            __syncwarp();
            if (lb > thr) continue;
            if constexpr (!CARRY) {  // plain: the popped node's record
                const uint32_t node = ea;
                const uint32_t fcn = KV(offsets)[node];
                if (fcn == 0) {
                    const uint2 rg = KV(ranges)[node];
                    ea = rg.x;
                    eb = rg.y;
                } else {
                    ea = fcn;
                    eb = 0xffffffffu;
                }
            }
            if (eb != 0xffffffffu) {
                // points [ea, eb): distances, candidates into the buffer
                for (uint32_t b = ea; b < eb; b += 32) {
                    const uint32_t i = b + lane;
                    double d = INFINITY;
                    bool cand = false;
                    if (i < eb) {
                        d = dist_pp(p[0], p[1], p[2], KV(xs)[i], KV(ys)[i], KV(zs)[i]);
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
                // internal: lower bounds and records of the 8 children, nearest pushed last
                const uint32_t fc = ea;
                const uint32_t cd = depth + 1;
                double clb = INFINITY;
                bool keep = false;
                uint32_t ca = 0, cb = 0;
                if (lane < 8) {
                    const uint32_t child = fc + lane;
                    clb = dist_po(p, KV(centers) + 3ull * child, s_radii[cd]);
                    if constexpr (CARRY) {
                        const uint32_t cfc = KV(offsets)[child];
                        const uint2 rg = KV(ranges)[child];
                        if (cfc && rg.y - rg.x > a.bucket) {
                            ca = cfc;
                            cb = 0xffffffffu;
                            keep = !(clb > thr);
                        } else {
                            ca = rg.x;
                            cb = rg.y;
                            keep = (rg.y > rg.x) && !(clb > thr);
                        }
                    } else {
                        ca = child;  // its record is read when it is popped
                        keep = !(clb > thr);
                    }
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
                    st_a[slot] = ca;
                    st_b[slot] = cb;
                    st_lb[slot] = clb;
                    st_depth[slot] = (uint8_t)cd;
                }
                __syncwarp();
                sp += nk;
            }
        }
        if (failed) set_err(a.err, kErrStackOverflow);
        if (nb > 0) merge();
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
    return (size_t)kKnnWarps * (per * 8 + (per + kKnnStack) * 4 + kKnnStack) + 16;
}

template <int LCAP>
cudaError_t launch_l(const KnnArgs& a, int grid, cudaStream_t s, bool carry) {
    const size_t smem = knn_smem<LCAP>();
    cudaError_t e;
    if (carry) {
        if ((e = cudaFuncSetAttribute(k_knn<LCAP, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem)) != cudaSuccess)
            return e;
        k_knn<LCAP, false, true><<<grid, kKnnThreads, smem, s>>>(a);
    } else {
        if ((e = cudaFuncSetAttribute(k_knn<LCAP, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem)) != cudaSuccess)
            return e;
        k_knn<LCAP, false, false><<<grid, kKnnThreads, smem, s>>>(a);
    }
    return cudaGetLastError();
}

// Table launch of the list kernel (the engine's kNN groups with 64 < k <= LCAP).
template <int LCAP>
cudaError_t launch_l_table(const DynGroup* d_grp, const uint32_t* order, uint32_t bucket, uint32_t* idx, double* d2,
                           uint32_t* counts, uint32_t* err, int grid, cudaStream_t s) {
    KnnArgs a{};
    a.grp = d_grp;
    a.bucket = bucket;
    a.order = order;
    a.idx = idx;
    a.d2 = d2;
    a.counts = counts;
    a.err = err;
    k_knn<LCAP, true><<<grid, kKnnThreads, knn_smem<LCAP>(), s>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Register kNN for k <= 64: one warp per query, the k best (distance, index)
// pairs held in registers as a sorted list (R = 1 or 2 entries per lane,
// element j = r * 32 + lane).  Leaf points that beat the k-th pair collect in a
// 32-entry shared buffer; a full buffer is merged into the list by a register
// bitonic sort + merge (xor shuffles, no shared-memory sort).  Children are judged with their ranges and first-child links loaded at
// expansion time, so empty leaves are never pushed and a popped entry needs no
// further dependent loads before its points are read.
// ---------------------------------------------------------------------------

template <int R>
struct RegList {
    double d[R];
    uint32_t i[R];
};

template <int R>
__device__ __forceinline__ void reglist_kth(const RegList<R>& L, uint32_t K, double& td, uint32_t& ti) {
    const int r = (int)(K - 1) >> 5, src = (int)(K - 1) & 31;
    double d = L.d[0];
    uint32_t i = L.i[0];
#pragma unroll
    for (int rr = 1; rr < R; ++rr)
        if (rr == r) {
            d = L.d[rr];
            i = L.i[rr];
        }
    td = __shfl_sync(0xffffffffu, d, src);
    ti = __shfl_sync(0xffffffffu, i, src);
}

// Compare-exchange with the lane `lane ^ j`: keep the smaller pair when
// `keep_min`, else the larger.
__device__ __forceinline__ void cx_xor(double& d, uint32_t& i, int j, bool keep_min) {
    const double pd = __shfl_xor_sync(0xffffffffu, d, j);
    const uint32_t pi = __shfl_xor_sync(0xffffffffu, i, j);
    const bool partner_less = pair_less(pd, pi, d, i);
    if (partner_less == keep_min) {
        d = pd;
        i = pi;
    }
}

// Ascending bitonic sort of one pair per lane (32 pairs).
__device__ __forceinline__ void warp_sort32(double& d, uint32_t& i) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) cx_xor(d, i, j, ((lane & j) == 0) == ((lane & k) == 0));
}

// Sort a bitonic sequence of 32 pairs (one per lane) ascending.
__device__ __forceinline__ void warp_bitonic_merge32(double& d, uint32_t& i) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) cx_xor(d, i, j, (lane & j) == 0);
}

// Merge 32 unsorted candidate pairs (one per lane, +inf for none) into the
// sorted register list, keeping the smallest 32 * R pairs.  For R = 2: the 32
// smallest of (upper half, candidates) are min(upper[l], sorted_cand[31 - l]),
// and the 64 smallest of everything are the lower half merged with those.
template <int R>
__device__ __forceinline__ void reglist_merge32(RegList<R>& L, double cd, uint32_t ci) {
    const int lane = threadIdx.x & 31;
    warp_sort32(cd, ci);
    const double rd = __shfl_sync(0xffffffffu, cd, 31 - lane);
    const uint32_t ri = __shfl_sync(0xffffffffu, ci, 31 - lane);
    double md = L.d[R - 1];
    uint32_t mi = L.i[R - 1];
    if (pair_less(rd, ri, md, mi)) {
        md = rd;
        mi = ri;
    }
    warp_bitonic_merge32(md, mi);
    if constexpr (R == 1) {
        L.d[0] = md;
        L.i[0] = mi;
    } else {
        // lower half L0 (ascending) against reversed M: min goes low, max goes high
        const double xd = __shfl_sync(0xffffffffu, md, 31 - lane);
        const uint32_t xi = __shfl_sync(0xffffffffu, mi, 31 - lane);
        double lo_d = L.d[0], hi_d = xd;
        uint32_t lo_i = L.i[0], hi_i = xi;
        if (pair_less(xd, xi, lo_d, lo_i)) {
            hi_d = lo_d;
            hi_i = lo_i;
            lo_d = xd;
            lo_i = xi;
        }
        warp_bitonic_merge32(lo_d, lo_i);
        warp_bitonic_merge32(hi_d, hi_i);
        L.d[0] = lo_d;
        L.i[0] = lo_i;
        L.d[1] = hi_d;
        L.i[1] = hi_i;
    }
}

struct KnnTableArgs {
    SearchReq single;        // the request of a single-cloud search (grp == null)
    const DynGroup* grp;     // sizes and request table of a batch group (device)
    uint64_t nq;             // queries of a single-request launch
    const uint32_t* order;   // visiting order (global query positions), or null
    uint32_t bucket;
    uint32_t* idx;
    double* d2;
    uint32_t* counts;
    uint32_t* err;
    double est;              // > 0: provisional k-th distance from the first range's density (factor), 0: off
    const unsigned long long* nq_dev;  // single-request launch: the query count in device memory (else nq)
};

// MULTI 0: one request in the kernel parameters; 1: a request table, the
// current request's cloud pointers in shared memory; 2: a request table whose
// requests are all on the cloud single.cv (kernel parameters)
#define KRQ(f) (MULTI ? reqs[ri].f : a.single.f)
#define KRQV(f) (MULTI == 1 ? s_view[warp].f : a.single.cv.f)
template <int R, int MULTI>
__global__ void __launch_bounds__(kKnnThreads, 8) k_knn_reg(KnnTableArgs a) {
    __shared__ uint32_t st_a[kKnnWarps][kKnnStack];   // leaf: first point; internal: first child
    __shared__ uint32_t st_b[kKnnWarps][kKnnStack];   // leaf: end point; internal: 0xffffffff
    __shared__ double st_lb[kKnnWarps][kKnnStack];
    __shared__ uint8_t st_depth[kKnnWarps][kKnnStack];
    __shared__ double s_rad[kKnnWarps][kMaxDepth + 1][3];
    __shared__ double s_bd[kKnnWarps][32];
    __shared__ uint32_t s_bi[kKnnWarps][32];
    __shared__ CloudView s_view[MULTI == 1 ? kKnnWarps : 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double (*s_radii)[3] = s_rad[warp];
    uint32_t cur_cloud = 0xffffffffu;
    uint32_t* sa = st_a[warp];
    uint32_t* sb = st_b[warp];
    double* sl = st_lb[warp];
    uint8_t* sd = st_depth[warp];
    const SearchReq* reqs = nullptr;
    uint32_t nreq = 1;
    uint64_t q0 = 0, nq = a.nq;
    if (MULTI) {
        reqs = a.grp->reqs;
        nreq = a.grp->nreq;
        q0 = a.grp->q_begin;
        nq = a.grp->nq;
    } else if (a.nq_dev) {
        nq = *a.nq_dev;
    }
    const uint64_t nwarps = (uint64_t)gridDim.x * kKnnWarps;
    for (uint64_t w = (uint64_t)blockIdx.x * kKnnWarps + warp; w < nq; w += nwarps) {
        const uint64_t qpos = q0 + w;
        const uint64_t q = a.order ? a.order[qpos] : qpos;  // global query position
        uint32_t ri = 0;
        if (MULTI) {  // the request whose positions contain q (q_begin ascending)
            uint32_t lo = 0, hi = nreq;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (reqs[mid].q_begin <= q) lo = mid;
                else hi = mid;
            }
            ri = lo;
        }
        if (KRQ(cloud_id) != cur_cloud) {
            __syncwarp();
            const double* gr = &KRQ(cv.geom)->radii[0][0];
            for (int t = lane; t < (kMaxDepth + 1) * 3; t += 32) (&s_radii[0][0])[t] = gr[t];
            if (MULTI == 1 && lane == 0) s_view[warp] = reqs[ri].cv;
            cur_cloud = KRQ(cloud_id);
            __syncwarp();
        }
        const uint32_t K = KRQ(k);
        const uint64_t ql = q - KRQ(q_begin);
        const double* qc = KRQ(centers);
        const double p[3] = {qc[3 * ql], qc[3 * ql + 1], qc[3 * ql + 2]};
        RegList<R> L;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            L.d[r] = INFINITY;
            L.i[r] = 0xffffffffu;
        }
        uint32_t nl = 0;
        double thr = INFINITY;
        uint32_t thr_i = 0xffffffffu;
        bool failed = false;
        uint32_t nb = 0;  // candidates waiting in the shared buffer
        double* bd = s_bd[warp];
        uint32_t* bi = s_bi[warp];
        // Provisional threshold: at the first point range the search reaches (the
        // query's own cell, nearest first), the squared radius holding about
        // `est` x k points at that cell's points per unit of xy area.  Nodes and
        // points beyond it are skipped; every point within it is still visited
        // (lower bounds never exceed distances), so if at least k points lie
        // within it the k best are exact, and otherwise the query runs again
        // without it.
        bool est_pending = a.est > 0.0, est_used = false;
        for (int attempt = 0; attempt < 2; ++attempt) {
        auto merge_buf = [&]() {
            const double cdv = (lane < (int)nb) ? bd[lane] : (double)INFINITY;
            const uint32_t civ = (lane < (int)nb) ? bi[lane] : 0xffffffffu;
            __syncwarp();
            reglist_merge32<R>(L, cdv, civ);
            nl = (nl + nb < K) ? nl + nb : K;
            nb = 0;
            if (nl == K) reglist_kth<R>(L, K, thr, thr_i);
        };
        // root (bound 0, linear_octree.hpp:904)
        {
            const uint32_t fc0 = KRQV(offsets)[0];
            const uint2 rg0 = KRQV(ranges)[0];
            const bool scan0 = fc0 == 0 || rg0.y - rg0.x <= a.bucket;
            if (lane == 0) {
                sa[0] = scan0 ? rg0.x : fc0;
                sb[0] = scan0 ? rg0.y : 0xffffffffu;
                sl[0] = 0.0;
                sd[0] = 0;
            }
        }
        __syncwarp();
        int sp = 1;
        while (sp > 0) {
            --sp;
            const uint32_t ea = sa[sp], eb = sb[sp];
            const double lb = sl[sp];
            const uint32_t depth = sd[sp];
            __syncwarp();
            if (lb > thr) continue;
            if (eb != 0xffffffffu) {
                if (est_pending) {
                    est_pending = false;
                    const double area = 4.0 * s_radii[depth][0] * s_radii[depth][1];
                    if (area > 0.0) {
                        thr = a.est * (double)K * area / (3.14159265358979323846 * (double)(eb - ea));
                        thr_i = 0xffffffffu;  // with the pair order this accepts d <= thr
                        est_used = true;
                    }
                }
                // leaf [ea, eb): candidates beat the k-th pair
                for (uint32_t b = ea; b < eb; b += 32) {
                    const uint32_t i = b + lane;
                    double d = INFINITY;
                    bool cand = false;
                    if (i < eb) {
                        d = dist_pp(p[0], p[1], p[2], KRQV(xs)[i], KRQV(ys)[i], KRQV(zs)[i]);
                        cand = pair_less(d, i, thr, thr_i);
                    }
                    uint32_t m = __ballot_sync(0xffffffffu, cand);
                    if (nb + __popc(m) > 32) {
                        merge_buf();
                        cand = cand && pair_less(d, i, thr, thr_i);
                        m = __ballot_sync(0xffffffffu, cand);
                    }
                    if (cand) {
                        const uint32_t slot = nb + __popc(m & lanemask_lt());
                        bd[slot] = d;
                        bi[slot] = i;
                    }
                    nb += __popc(m);
                    __syncwarp();
                }
                continue;
            }
            // internal: judge the 8 children (bound, first child / range), nearest on top
            const uint32_t fc = ea;
            const uint32_t cd = depth + 1;
            double clb = INFINITY;
            bool keep = false;
            uint32_t ca = 0, cb = 0;
            if (lane < 8) {
                const uint32_t child = fc + lane;
                clb = dist_po(p, KRQV(centers) + 3ull * child, s_radii[cd]);
                const uint32_t cfc = KRQV(offsets)[child];
                const uint2 rg = KRQV(ranges)[child];
                if (cfc && rg.y - rg.x > a.bucket) {
                    ca = cfc;
                    cb = 0xffffffffu;
                    keep = !(clb > thr);
                } else {
                    // a leaf, or a small subtree scanned as one range: extra points can only be
                    // rejected by the k-th pair, so the k best pairs are unchanged
                    ca = rg.x;
                    cb = rg.y;
                    keep = (rg.y > rg.x) && !(clb > thr);  // an empty leaf holds no candidate
                }
            }
            const uint32_t km = __ballot_sync(0xffffffffu, keep) & 0xffu;
            const int nk = __popc(km);
            if (sp + nk > kKnnStack) {
                failed = true;
                break;
            }
            int pos = 0;
#pragma unroll
            for (int o = 0; o < 8; ++o) {
                const double ol = __shfl_sync(0xffffffffu, clb, o);
                const bool ok = (km >> o) & 1u;
                if (ok && o != lane && ((ol > clb) || (ol == clb && o > lane))) ++pos;
            }
            if (keep) {
                const int slot = sp + pos;
                sa[slot] = ca;
                sb[slot] = cb;
                sl[slot] = clb;
                sd[slot] = (uint8_t)cd;
            }
            __syncwarp();
            sp += nk;
        }
        if (nb) merge_buf();
        if (!(est_used && nl < K) || failed) break;
        // fewer than k points within the provisional threshold: again, without it
#pragma unroll
        for (int r = 0; r < R; ++r) {
            L.d[r] = INFINITY;
            L.i[r] = 0xffffffffu;
        }
        nl = 0;
        thr = INFINITY;
        thr_i = 0xffffffffu;
        est_used = false;
        __syncwarp();
        }
        if (failed) set_err(a.err, kErrStackOverflow);
        const uint64_t o = KRQ(out_begin) + ql * (uint64_t)K;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t j = (uint32_t)(r * 32 + lane);
            if (j < K) {
                a.idx[o + j] = (j < nl) ? L.i[r] : 0xffffffffu;
                a.d2[o + j] = (j < nl) ? L.d[r] : (double)INFINITY;
            }
        }
        if (lane == 0 && a.counts) a.counts[q] = nl;
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Group kNN (k <= 64): kGrpQ (4) curve-ordered queries per warp share one walk.
//
// Consecutive queries along the curve are a few metres apart, so the octants
// their searches need overlap almost entirely: 4 of them visit ~4.7 internal
// nodes per query (8: ~2.9) where one query alone visits ~14 (10M-point tile,
// k = 50).  Groups of 4 rather than 8 halve the shared memory per warp, so 28
// warps fit on an SM instead of 16, which this latency-bound walk needs more.
// The warp walks the tree once for its group, nearest first by the smallest
// lower bound of the group; a child is pushed with the mask of queries that
// accept it and, per query, its lower bound rounded down to FP16 (a popped
// entry is skipped for a query whose threshold has since dropped below it; the
// rounding only keeps entries).  At an internal node 32 / kGrpQ lanes per
// query judge the 8 children.  A range (leaf, or subtree of at most `bucket`
// points) is tested transposed: the lanes hold 32 consecutive points and test
// them against one accepting query at a time, and the query's candidates
// (pairs that beat its k-th pair) go to its own 32-entry buffer in shared
// memory; a full buffer is merged into the query's sorted list (in shared
// memory, R x 32 pairs) by the warp with the same register bitonic merge as
// k_knn_reg.  Provisional thresholds: a warp takes `chunk` consecutive groups
// at a time, and every group after the first of a run starts each query at
// kGrpSeed x the largest k-th distance of the group before it (the k-th
// distance varies slowly along the curve: this holds ~1.4 k points where the
// density estimate of k_knn_reg holds several times more, so half the
// candidates and merges go; longer runs widen the stretch of the curve that
// the warps work on at once, which costs L2 hits).  Every kKnnHeadStride-th
// group is a head: heads are handed out first and take k_knn_reg's density
// estimate from the first range each query reaches; the first group of a run
// (and each group handed out alone at the end) starts from the nearest head
// of its request that has finished, or from the density estimate when none
// has (no group waits for a head).  F32: range points are first tested in FP32
// (centre-relative copies) against a per-query FP32 bound of the threshold
// (knn_f32_threshold); only points not rejected take the FP64 distance.  A query that ends with fewer than k pairs
// inside its provisional threshold, and every query of a group whose stack
// overflowed, is appended to a fallback list that k_knn_reg completes exactly.
// ---------------------------------------------------------------------------

constexpr int kGrpQ = (int)kKnnGroupQueries;  // queries per warp: 4 or 8 (query masks are 8 bits)
// blocks as shared memory allows: ~12.5 KB per warp of 8 queries, ~6.5 KB per warp of 4
// (8 blocks of 4 warps: 32 warps per SM at up to 64 registers)
constexpr int kGrpWarps = kGrpQ == 8 ? 2 : 4;
constexpr int kGrpMinBlocks = 8;
constexpr int kGrpThreads = 32 * kGrpWarps;
constexpr int kGrpStack = 88;
// provisional threshold / previous group's largest k-th distance (10M-point
// tile, k = 50: 1.15 -> 4.28 ms, 1.2 -> 4.04, 1.3 -> 3.83, 1.4 -> 3.78, 1.5 -> 3.79;
// results are the same for every factor: a threshold too small hands the query back)
constexpr double kGrpSeed = 1.4;
static_assert(kKnnHeadStride >= 2, "the groups between heads are numbered modulo kKnnHeadStride - 1");

struct KnnGroupArgs {
    SearchReq single;                 // one request (grp == null)
    const DynGroup* grp;              // a batch group: sizes and requests on the device
    uint64_t packets;                 // single: groups of kGrpQ queries
    const uint32_t* order;            // visiting order (global query positions)
    uint32_t bucket;
    uint32_t* idx;
    double* d2;
    uint32_t* counts;
    uint32_t* err;
    double est;                       // provisional-threshold factor (0: off, also no seeding)
    uint32_t* packet_ctr;             // [0] runs of `chunk` groups, [1] single groups at the end, [2] heads
    uint32_t chunk;                   // consecutive groups per fetch (>= 1)
    uint32_t head_stride;             // S > 1: every S-th group is a head, taken first (0: no heads)
    double* head_kth;                 // per head: the largest k-th distance it found (NaN: not yet, < 0: none)
    unsigned long long* stats;        // FP32 filter: point tests, FP64 tests, band hits (may be null)
    uint32_t* fb_list;                // queries left to k_knn_reg (global positions; a batch group's
                                      // entries start at its q_begin)
    unsigned long long* fb_count;
};

// FP32 filter of the group kNN: a point whose FP32 squared distance D_f to
// the query exceeds the returned value has an exact squared distance above
// thr.  Per axis a = p - centre (|a| <= A, the box radius) and b = q - centre
// (|b| <= B) are each rounded once to FP32 from their FP64 differences, and
// delta_f = fl32(a_f - b_f); with u = 2^-24, |delta_f - delta| <= 1.0002 u
// (A + B + |delta|).  For D <= thr (|delta| <= s = sqrt thr, M = A + B + s):
// |sum delta_f^2 - D| <= 2 * 1.0002 u M sqrt(3) s + 3.0012 u^2 M^2, and the
// FP32 product and two fused adds add at most 3.0001 u sum delta_f^2 <=
// 3.0001 u (s + 1.733 u M)^2.  The threshold is thr plus twice that bound,
// rounded up to FP32.  ab = A + B.
__device__ __forceinline__ float knn_f32_threshold(double thr, double ab) {
    if (!(thr < (double)INFINITY)) return INFINITY;
    const double u = 5.9604644775390625e-08;  // 2^-24
    const double sr = sqrt(thr) * (1.0 + 1.0e-12);
    const double M = ab + sr;
    const double t = sr + 1.74 * u * M;
    const double err = 3.47 * u * M * sr + 3.01 * u * u * M * M + 3.01 * u * t * t;
    return __double2float_ru(thr + 2.0 * err);
}

template <int R, int MULTI, bool F32>
__global__ void __launch_bounds__(kGrpThreads, kGrpMinBlocks) k_knn_group(KnnGroupArgs a) {
    constexpr int G = kGrpQ;
    constexpr int LC = 32 * R;
    __shared__ double s_ld[kGrpWarps][G][LC];
    __shared__ uint32_t s_li[kGrpWarps][G][LC];
    __shared__ double s_bd[kGrpWarps][G][32];
    __shared__ uint32_t s_bi[kGrpWarps][G][32];
    __shared__ double s_q[kGrpWarps][G][3];
    __shared__ double s_thr[kGrpWarps][G];
    __shared__ uint32_t s_thri[kGrpWarps][G];
    __shared__ uint32_t s_nl[kGrpWarps][G];
    __shared__ uint32_t s_nb[kGrpWarps][G];
    __shared__ uint32_t s_qg[kGrpWarps][G];
    // FP32 filter: query - box centre in FP32 with the query's FP32 threshold in w,
    // and the query's A + B (box radius + |query - centre|_inf) for new thresholds
    __shared__ float4 s_qf[F32 ? kGrpWarps : 1][G];
    __shared__ double s_qab[F32 ? kGrpWarps : 1][G];
    unsigned long long f_tests = 0, f_64 = 0, f_band = 0;
    __shared__ uint32_t st_a[kGrpWarps][kGrpStack];
    __shared__ uint32_t st_b[kGrpWarps][kGrpStack];
    __shared__ __half st_lb[kGrpWarps][kGrpStack][G];  // per-query bounds, rounded down to FP16
    __shared__ uint8_t st_d[kGrpWarps][kGrpStack];
    __shared__ uint8_t st_m[kGrpWarps][kGrpStack];
    // level radii: per warp for a table of clouds, once per block for one cloud
    __shared__ double s_rad[MULTI == 1 ? kGrpWarps : 1][kMaxDepth + 1][3];
    __shared__ CloudView s_view[MULTI == 1 ? kGrpWarps : 1];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double (*s_radii)[3] = s_rad[MULTI == 1 ? warp : 0];
    if (MULTI != 1) {
        const double* gr = &a.single.cv.geom->radii[0][0];
        for (int t = threadIdx.x; t < (kMaxDepth + 1) * 3; t += kGrpThreads) (&s_rad[0][0][0])[t] = gr[t];
        __syncthreads();
    }
    double (*ld)[LC] = s_ld[warp];
    uint32_t (*li)[LC] = s_li[warp];
    double (*bd)[32] = s_bd[warp];
    uint32_t (*bi)[32] = s_bi[warp];
    double (*qs)[3] = s_q[warp];
    double* thr = s_thr[warp];
    uint32_t* thri = s_thri[warp];
    uint32_t* nls = s_nl[warp];
    uint32_t* nbs = s_nb[warp];
    uint32_t* sa = st_a[warp];
    uint32_t* sb = st_b[warp];
    __half (*slb)[G] = st_lb[warp];
    uint8_t* sdp = st_d[warp];
    uint8_t* smk = st_m[warp];
    uint32_t cur_cloud = 0xffffffffu;
    const SearchReq* reqs = nullptr;
    uint32_t nreq = 1;
    // query positions and group indices of a launch fit 32 bits (positions are u32 in the order arrays)
    uint32_t packets = (uint32_t)a.packets;
    uint32_t fb_base = 0;  // the fallback entries of a batch group start at its first position
    if (MULTI) {
        reqs = a.grp->reqs;
        nreq = a.grp->nreq;
        packets = (uint32_t)a.grp->packets;
        fb_base = (uint32_t)a.grp->q_begin;
    }
    // lane roles at an internal node: LPQ lanes per query qj, CPL children each
    constexpr int LPQ = 32 / G, CPL = 8 / LPQ;
    static_assert(G == 4 || G == 8, "4 or 8 queries per warp");
    const int qj = lane / LPQ, cs = lane % LPQ;
    // heads (every S-th group) go out first, one at a time; the other groups are
    // slots: slot s is the s-th group that is not a head (every group without heads)
    const uint32_t S = a.head_stride;
    const uint32_t n_heads = S ? (packets + S - 1) / S : 0;
    const uint32_t slots = packets - n_heads;
    bool heads_left = n_heads != 0;
    // slots [0, p_chunked) go out in chunks, the rest one at a time
    const uint32_t nw = gridDim.x * kGrpWarps;
    const uint32_t chunk = a.chunk;
    const uint32_t p_chunked = (chunk > 1 && slots > 2 * nw) ? (slots - 2 * nw) / chunk * chunk : 0;
    uint32_t next = 0, chunk_end = 0;
    // seed: the previous group's largest k-th distance (< 0: none), its slot and request
    double seed_thr = -1.0;
    uint32_t seed_slot = 0;
    uint32_t seed_ri = 0;

    for (;;) {
        uint32_t slot = 0xffffffffu;  // the head's group index when a head
        bool head = false;
        if (heads_left) {
            uint32_t h = 0;
            if (lane == 0) h = atomicAdd(&a.packet_ctr[2], 1u);
            h = __shfl_sync(0xffffffffu, h, 0);
            if (h < n_heads) head = true, slot = h;
            else heads_left = false;
        }
        if (!head) {
            if (next < chunk_end) {
                slot = next++;
            } else {
                uint32_t v = 0;
                if (lane == 0) v = atomicAdd(&a.packet_ctr[0], 1u);
                v = __shfl_sync(0xffffffffu, v, 0);
                const uint64_t c0 = (uint64_t)v * chunk;
                if (c0 < p_chunked) {
                    slot = (uint32_t)c0;
                    next = slot + 1;
                    chunk_end = slot + chunk;
                } else {
                    uint32_t s = 0;
                    if (lane == 0) s = atomicAdd(&a.packet_ctr[1], 1u);
                    s = __shfl_sync(0xffffffffu, s, 0);
                    if ((uint64_t)p_chunked + s >= slots) break;
                    slot = p_chunked + s;
                    next = chunk_end = 0;
                }
            }
            if (slot >= slots) break;
        }
        const uint32_t packet = head ? slot * S : !S ? slot : slot + slot / (S - 1) + 1;
        uint32_t ri = 0;
        if (MULTI) {  // the request of this group (packet_begin ascending over the table)
            uint32_t lo = 0, hi = nreq;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (reqs[mid].packet_begin <= packet) lo = mid;
                else hi = mid;
            }
            ri = lo;
        }
        if (MULTI == 1 && reqs[ri].cloud_id != cur_cloud) {  // this warp's level radii and cloud follow the group's
            __syncwarp();
            const double* gr = &reqs[ri].cv.geom->radii[0][0];
            for (int t = lane; t < (kMaxDepth + 1) * 3; t += 32) (&s_radii[0][0])[t] = gr[t];
            if (lane == 0) s_view[warp] = reqs[ri].cv;
            cur_cloud = reqs[ri].cloud_id;
            __syncwarp();
        }
        const uint32_t K = KRQ(k);
        const uint32_t q_begin = (uint32_t)KRQ(q_begin);
        const uint32_t pos0 = q_begin + (uint32_t)G * (packet - (uint32_t)KRQ(packet_begin));
        const uint32_t q_end = (uint32_t)KRQ(q_end);
        // seed: the group before this one in the warp's run, else (between heads) the
        // nearest head of the same request
        // heads start from the density estimate
        double seed = (a.est > 0.0 && !head && seed_thr >= 0.0 && slot == seed_slot + 1 && ri == seed_ri)
                          ? seed_thr : -1.0;
        if (seed < 0.0 && a.est > 0.0 && S && !head) {
            const uint32_t pb = (uint32_t)KRQ(packet_begin);
            const uint32_t pe = pb + (uint32_t)((KRQ(q_end) - KRQ(q_begin) + G - 1) / G);
            const uint32_t hlo = packet / S, hhi = hlo + 1;  // heads hlo S < packet < hhi S
            const bool lo_ok = hlo * S >= pb, hi_ok = hhi < n_heads && hhi * S < pe;
            const bool use_hi = hi_ok && (!lo_ok || hhi * S - packet < packet - hlo * S);
            // a head not finished yet reads NaN: no seed (nothing waits for it)
            if (use_hi || lo_ok) seed = __ldcg(&a.head_kth[use_hi ? hhi : hlo]);
            if (!(seed >= 0.0)) seed = -1.0;
        }
        const bool seeded = seed >= 0.0;
        // lanes j < G: load query j, reset its state
        bool valid = false;
        if (lane < G) {
            const uint64_t pos = pos0 + lane;
            valid = pos < q_end;
            const uint64_t q = valid ? (uint64_t)a.order[pos] : q_begin;
            const uint64_t ql = q - q_begin;
            const double* qc = KRQ(centers);
            qs[lane][0] = qc[3 * ql];
            qs[lane][1] = qc[3 * ql + 1];
            qs[lane][2] = qc[3 * ql + 2];
            thr[lane] = seeded ? kGrpSeed * seed : (double)INFINITY;
            thri[lane] = 0xffffffffu;  // with the pair order a provisional threshold accepts d <= thr
            nls[lane] = 0;
            nbs[lane] = 0;
            s_qg[warp][lane] = (uint32_t)q;
            if constexpr (F32) {
                const BoxD* bx = KRQV(box);
                const double bqx = dsub(qc[3 * ql], bx->center[0]);
                const double bqy = dsub(qc[3 * ql + 1], bx->center[1]);
                const double bqz = dsub(qc[3 * ql + 2], bx->center[2]);
                const double A = smax(smax(bx->radii[0], bx->radii[1]), bx->radii[2]);
                const double B = smax(smax(fabs(bqx), fabs(bqy)), fabs(bqz));
                const double ab = (A + B) * (1.0 + 1.0e-12);
                s_qab[warp][lane] = ab;
                s_qf[warp][lane] = make_float4((float)bqx, (float)bqy, (float)bqz, knn_f32_threshold(thr[lane], ab));
            }
        }
        for (int t = lane; t < G * LC; t += 32) {
            (&ld[0][0])[t] = INFINITY;
            (&li[0][0])[t] = 0xffffffffu;
        }
        const uint32_t vm = __ballot_sync(0xffffffffu, valid) & ((1u << G) - 1u);
        uint32_t est_pend = (a.est > 0.0 && !seeded) ? vm : 0u, est_used = seeded ? vm : 0u;
        bool failed = false;

        // Merge query j's buffer (nb > 0 pairs) into its list (warp-uniform call).
        auto merge = [&](int j, uint32_t nb) {
            const double cdv = (lane < (int)nb) ? bd[j][lane] : (double)INFINITY;
            const uint32_t civ = (lane < (int)nb) ? bi[j][lane] : 0xffffffffu;
            RegList<R> L;
            if (nls[j] == 0) {  // an empty list (every entry +inf): the sorted candidates are the merge
                double sd = cdv;
                uint32_t si = civ;
                warp_sort32(sd, si);
                L.d[0] = sd;
                L.i[0] = si;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    L.d[r] = INFINITY;
                    L.i[r] = 0xffffffffu;
                }
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    L.d[r] = ld[j][r * 32 + lane];
                    L.i[r] = li[j][r * 32 + lane];
                }
                reglist_merge32<R>(L, cdv, civ);
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                ld[j][r * 32 + lane] = L.d[r];
                li[j][r * 32 + lane] = L.i[r];
            }
            uint32_t nl = nls[j] + nb;
            if (nl > K) nl = K;
            double td = 0.0;
            uint32_t ti = 0;
            if (nl == K) reglist_kth<R>(L, K, td, ti);
            __syncwarp();
            if (lane == 0) {
                nls[j] = nl;
                nbs[j] = 0;
                if (nl == K) {
                    thr[j] = td;
                    thri[j] = ti;
                    if constexpr (F32) s_qf[warp][j].w = knn_f32_threshold(td, s_qab[warp][j]);
                }
            }
            __syncwarp();
        };

        // root (bound 0)
        {
            const uint32_t fc0 = KRQV(offsets)[0];
            const uint2 rg0 = KRQV(ranges)[0];
            const bool scan0 = fc0 == 0 || rg0.y - rg0.x <= a.bucket;
            if (lane == 0) {
                sa[0] = scan0 ? rg0.x : fc0;
                sb[0] = scan0 ? rg0.y : 0xffffffffu;
                sdp[0] = 0;
                smk[0] = (uint8_t)vm;
            }
            if (lane < G) slb[0][lane] = __float2half_rz(0.0f);
        }
        __syncwarp();
        int sp = vm ? 1 : 0;
        while (sp > 0) {
            --sp;
            const uint32_t ea = sa[sp], eb = sb[sp];
            const uint32_t depth = sdp[sp];
            bool act = false;
            if (lane < G) act = ((smk[sp] >> lane) & 1u) && !((double)__half2float(slb[sp][lane]) > thr[lane]);
            const uint32_t m = __ballot_sync(0xffffffffu, act) & ((1u << G) - 1u);
            __syncwarp();
            if (!m) continue;
            if (eb != 0xffffffffu) {
                // a range [ea, eb)
                const uint32_t pend = est_pend & m;
                if (pend) {
                    const double area = 4.0 * s_radii[depth][0] * s_radii[depth][1];
                    if (area > 0.0) {
                        if (lane < G && ((pend >> lane) & 1u)) {
                            thr[lane] = a.est * (double)K * area / (3.14159265358979323846 * (double)(eb - ea));
                            thri[lane] = 0xffffffffu;  // with the pair order this accepts d <= thr
                            if constexpr (F32) s_qf[warp][lane].w = knn_f32_threshold(thr[lane], s_qab[warp][lane]);
                        }
                        est_used |= pend;
                    }
                    est_pend &= ~pend;
                    __syncwarp();
                }
                for (uint32_t b = ea; b < eb; b += 32) {
                    const uint32_t i = b + lane;
                    const bool in = i < eb;
                    double px = 0.0, py = 0.0, pz = 0.0;
                    float4 pf = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    bool have64 = !F32;  // the FP32 form reads FP64 coordinates only for points near a threshold
                    if (in) {
                        if constexpr (F32) {
                            pf = KRQV(crel)[i];
                        } else {
                            px = KRQV(xs)[i];
                            py = KRQV(ys)[i];
                            pz = KRQV(zs)[i];
                        }
                    }
                    if (F32 && lane == 0) f_tests += (unsigned long long)__popc(m) * ((eb - b < 32u) ? (eb - b) : 32u);
                    uint32_t rem = m;
                    while (rem) {
                        const int j = __ffs(rem) - 1;
                        rem &= rem - 1;
                        double d = (double)INFINITY;
                        bool cand = false;
                        if constexpr (F32) {
                            const float4 q4 = s_qf[warp][j];
                            const float dx = pf.x - q4.x, dy = pf.y - q4.y, dz = pf.z - q4.z;
                            const float df = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
                            if (in && !(df > q4.w)) {  // near the threshold or inside: the exact FP64 test
                                if (!have64) {
                                    px = KRQV(xs)[i];
                                    py = KRQV(ys)[i];
                                    pz = KRQV(zs)[i];
                                    have64 = true;
                                }
                                d = dist_pp(qs[j][0], qs[j][1], qs[j][2], px, py, pz);
                                cand = pair_less(d, i, thr[j], thri[j]);
                                ++f_64;
                                f_band += cand ? 0u : 1u;
                            }
                        } else {
                            d = dist_pp(qs[j][0], qs[j][1], qs[j][2], px, py, pz);
                            cand = in && pair_less(d, i, thr[j], thri[j]);
                        }
                        uint32_t hb = __ballot_sync(0xffffffffu, cand);
                        if (!hb) continue;
                        uint32_t nb = nbs[j];
                        if (nb + __popc(hb) > 32u) {
                            merge(j, nb);
                            nb = 0;
                            cand = cand && pair_less(d, i, thr[j], thri[j]);
                            hb = __ballot_sync(0xffffffffu, cand);
                        }
                        if (cand) {
                            const uint32_t slot = nb + __popc(hb & lanemask_lt());
                            bd[j][slot] = d;
                            bi[j][slot] = i;
                        }
                        __syncwarp();
                        if (lane == 0) nbs[j] = nb + __popc(hb);
                        __syncwarp();
                    }
                }
                continue;
            }
            // internal node: lane (qj, cs) judges children cs CPL .. cs CPL + CPL - 1 for query qj
            const uint32_t fc = ea;
            const uint32_t cd = depth + 1;
            const bool qa = (m >> qj) & 1u;
            double lb[CPL];
            bool kp[CPL];
            uint32_t B[CPL];
            double v[CPL];
#pragma unroll
            for (int w = 0; w < CPL; ++w) {
                lb[w] = INFINITY;
                kp[w] = false;
            }
            if (qa) {
                const double* c0 = KRQV(centers) + 3ull * (fc + CPL * cs);
                const double t = thr[qj];
#pragma unroll
                for (int w = 0; w < CPL; ++w) {
                    lb[w] = dist_po(qs[qj], c0 + 3 * w, s_radii[cd]);
                    kp[w] = !(lb[w] > t);
                }
            }
            // smallest accepting bound per child, over the lanes judging the same children
#pragma unroll
            for (int w = 0; w < CPL; ++w) {
                B[w] = __ballot_sync(0xffffffffu, kp[w]);
                v[w] = kp[w] ? lb[w] : (double)INFINITY;
            }
#pragma unroll
            for (int off = LPQ; off < 32; off <<= 1)
#pragma unroll
                for (int w = 0; w < CPL; ++w) v[w] = fmin(v[w], __shfl_xor_sync(0xffffffffu, v[w], off));
            // lane c < 8: child c's query mask, bound and record
            const int cc = lane & 7;
            double key = INFINITY;
            uint32_t Bw = 0;
#pragma unroll
            for (int w = 0; w < CPL; ++w) {
                const double x = __shfl_sync(0xffffffffu, v[w], cc / CPL);
                if (cc % CPL == w) {
                    key = x;
                    Bw = B[w];
                }
            }
            uint32_t cm = 0;
            uint32_t ca = 0, cb = 0;
            if (lane < 8) {
#pragma unroll
                for (int j = 0; j < G; ++j) cm |= ((Bw >> (LPQ * j + cc / CPL)) & 1u) << j;
                const uint32_t child = fc + lane;
                const uint32_t cfc = KRQV(offsets)[child];
                const uint2 rg = KRQV(ranges)[child];
                if (cfc && rg.y - rg.x > a.bucket) {
                    ca = cfc;
                    cb = 0xffffffffu;
                } else {
                    ca = rg.x;
                    cb = rg.y;
                    if (rg.y == rg.x) cm = 0;  // an empty leaf holds no candidate
                }
            } else {
                key = INFINITY;
            }
            const uint32_t pushm = __ballot_sync(0xffffffffu, lane < 8 && cm != 0);
            const int np = __popc(pushm);
            if (sp + np > kGrpStack) {
                failed = true;
                break;
            }
            // nearest on top: slot below every farther (or equal and higher octant) child
            int pos = 0;
#pragma unroll
            for (int o = 0; o < 8; ++o) {
                const double ol = __shfl_sync(0xffffffffu, key, o);
                if (((pushm >> o) & 1u) && o != lane && ((ol > key) || (ol == key && o > lane))) ++pos;
            }
            const int slot = sp + pos;
            if (lane < 8 && cm != 0) {
                sa[slot] = ca;
                sb[slot] = cb;
                sdp[slot] = (uint8_t)cd;
                smk[slot] = (uint8_t)cm;
            }
            // per-query bounds of the pushed children, rounded down
#pragma unroll
            for (int w = 0; w < CPL; ++w) {
                const int c = CPL * cs + w;
                const int sw = __shfl_sync(0xffffffffu, slot, c);
                if (kp[w] && ((pushm >> c) & 1u)) slb[sw][qj] = __float2half_rd(__double2float_rd(lb[w]));
            }
            __syncwarp();
            sp += np;
        }
        __syncwarp();
        // flush the buffers, then write each query's pairs or hand it to the fallback
        uint32_t rem = vm;
        while (rem) {
            const int j = __ffs(rem) - 1;
            rem &= rem - 1;
            const uint32_t nb = nbs[j];
            if (nb) merge(j, nb);
            const uint32_t nl = nls[j];
            const uint64_t q = s_qg[warp][j];
            if (failed || (((est_used >> j) & 1u) && nl < K)) {
                if (lane == 0) {
                    const unsigned long long f = atomicAdd(a.fb_count, 1ull);
                    a.fb_list[fb_base + f] = (uint32_t)q;
                }
                continue;
            }
            const uint64_t o = KRQ(out_begin) + (q - q_begin) * (uint64_t)K;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t jj = (uint32_t)(r * 32 + lane);
                if (jj < K) {
                    a.idx[o + jj] = (jj < nl) ? li[j][jj] : 0xffffffffu;
                    a.d2[o + jj] = (jj < nl) ? ld[j][jj] : (double)INFINITY;
                }
            }
            if (lane == 0 && a.counts) a.counts[q] = nl;
        }
        // seed of the next group: the largest k-th distance of the queries that found k pairs
        double mx = -1.0;
        if (lane < G && ((vm >> lane) & 1u) && !failed && nls[lane] == K) mx = thr[lane];
#pragma unroll
        for (int off = 4; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        mx = __shfl_sync(0xffffffffu, mx, 0);
        seed_thr = mx;
        seed_slot = head ? 0xfffffffeu : slot;  // a head seeds no slot of the run
        seed_ri = ri;
        if (head && lane == 0) __stcg(&a.head_kth[slot], mx);
        __syncwarp();
    }
    if constexpr (F32) {
        if (a.stats) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                f_64 += __shfl_xor_sync(0xffffffffu, f_64, off);
                f_band += __shfl_xor_sync(0xffffffffu, f_band, off);
            }
            if (lane == 0) {
                atomicAdd(&a.stats[0], f_tests);
                atomicAdd(&a.stats[1], f_64);
                atomicAdd(&a.stats[2], f_band);
            }
        }
    }
}

// Blocks per SM of a group-kNN instantiation (its shared memory sets it).
template <int R, int MULTI, bool F32>
int group_blocks_per_sm() {
    static int per = 0;
    if (per == 0) {
        int v = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_knn_group<R, MULTI, F32>, kGrpThreads, 0) !=
            cudaSuccess)
            v = 1;
        per = v > 0 ? v : 1;
    }
    return per;
}

// blocks_per_sm > 0 caps the resident blocks (room for a kernel running beside it).
template <int R, int MULTI, bool F32>
cudaError_t launch_group(const KnnGroupArgs& g, int sms, cudaStream_t s, int blocks_per_sm = 0) {
    int per = group_blocks_per_sm<R, MULTI, F32>();
    if (blocks_per_sm > 0 && blocks_per_sm < per) per = blocks_per_sm;
    uint64_t grid = (uint64_t)sms * per;
    if (!g.grp) {
        const uint64_t want = (g.packets + kGrpWarps - 1) / kGrpWarps;
        if (want < grid) grid = want;
    }
    if (grid == 0) return cudaSuccess;
    k_knn_group<R, MULTI, F32><<<(int)grid, kGrpThreads, 0, s>>>(g);
    return cudaGetLastError();
}

// The group search of a launch.  With seeding, every kKnnHeadStride-th group
// is a head: the heads go out first and start from the density estimate; every
// other group starts from its run's previous group or, when it leads its run,
// from the nearest head that has finished.  packet_ctr holds 3 counters (zeroed);
// head_kth one double per head, set to NaN here.  fp32: the FP32-filter form
// (every cloud of the launch has its centre-relative FP32 copy).
template <int R, int MULTI>
cudaError_t launch_group_seeded(KnnGroupArgs g, int sms, cudaStream_t s, int blocks_per_sm, double* head_kth,
                                size_t head_bytes, bool fp32) {
    g.head_stride = (g.est > 0.0 && head_kth) ? kKnnHeadStride : 0;
    g.head_kth = head_kth;
    if (g.head_stride) {
        const cudaError_t e = cudaMemsetAsync(head_kth, 0xff, head_bytes, s);
        if (e != cudaSuccess) return e;
    }
    if (fp32) return launch_group<R, MULTI, true>(g, sms, s, blocks_per_sm);
    return launch_group<R, MULTI, false>(g, sms, s, blocks_per_sm);
}

int sm_count_k(int device) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v;
}

}  // namespace

cudaError_t launch_knn_table(int device, cudaStream_t s, const DynGroup* d_grp, const SearchReq* single, uint64_t nq,
                             uint32_t kmax, const uint32_t* d_order, uint32_t bucket, uint32_t* d_idx, double* d_d2,
                             uint32_t* d_counts, uint32_t* d_err, int blocks_per_sm, double est) {
    if (!d_grp && nq == 0) return cudaSuccess;
    KnnTableArgs a{};
    a.single = single ? *single : SearchReq{};
    a.grp = d_grp;
    a.nq = nq;
    a.order = d_order;
    a.bucket = bucket;
    a.idx = d_idx;
    a.d2 = d_d2;
    a.counts = d_counts;
    a.err = d_err;
    a.est = est;
    const int sms = sm_count_k(device);
    const uint64_t cap = (uint64_t)sms * (blocks_per_sm > 0 ? blocks_per_sm : 16);
    const uint64_t want = d_grp ? cap : (nq + kKnnWarps - 1) / kKnnWarps;
    const int grid = (int)(want < cap ? want : cap);
    if (d_grp) {
        if (kmax > 64) {  // the shared-memory list kernel, blocks per SM as its list fits
            auto lgrid = [&](size_t smem) { return sms * (int)std::max<size_t>(1, (224u << 10) / (smem + 3072)); };
            if (kmax <= 128) return launch_l_table<128>(d_grp, d_order, bucket, d_idx, d_d2, d_counts, d_err,
                                                        lgrid(knn_smem<128>()), s);
            if (kmax <= 256) return launch_l_table<256>(d_grp, d_order, bucket, d_idx, d_d2, d_counts, d_err,
                                                        lgrid(knn_smem<256>()), s);
            if (kmax <= 512) return launch_l_table<512>(d_grp, d_order, bucket, d_idx, d_d2, d_counts, d_err,
                                                        lgrid(knn_smem<512>()), s);
            return launch_l_table<1024>(d_grp, d_order, bucket, d_idx, d_d2, d_counts, d_err, lgrid(knn_smem<1024>()),
                                        s);
        }
        if (single) {  // every request of the group on the cloud single->cv
            if (kmax <= 32) k_knn_reg<1, 2><<<grid, kKnnThreads, 0, s>>>(a);
            else k_knn_reg<2, 2><<<grid, kKnnThreads, 0, s>>>(a);
        } else {
            if (kmax <= 32) k_knn_reg<1, 1><<<grid, kKnnThreads, 0, s>>>(a);
            else k_knn_reg<2, 1><<<grid, kKnnThreads, 0, s>>>(a);
        }
    } else {
        if (kmax <= 32) k_knn_reg<1, 0><<<grid, kKnnThreads, 0, s>>>(a);
        else k_knn_reg<2, 0><<<grid, kKnnThreads, 0, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_knn_group_table(int device, cudaStream_t s, const DynGroup* d_grp, DynGroup* d_fb,
                                   const SearchReq* single, uint32_t kmax, const uint32_t* d_order, uint32_t bucket,
                                   uint32_t* d_idx, double* d_d2, uint32_t* d_counts, uint32_t* d_err,
                                   uint32_t* d_packet_ctr, uint32_t* d_fb_list, double est, uint32_t chunk,
                                   int blocks_per_sm, double* d_head_kth, size_t head_bytes, bool fp32,
                                   unsigned long long* d_stats) {
    if (kmax > 64) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = cudaMemsetAsync(d_packet_ctr, 0, 12, s)) != cudaSuccess) return e;
    KnnGroupArgs g{};
    g.single = single ? *single : SearchReq{};
    g.grp = d_grp;
    g.order = d_order;
    g.bucket = bucket;
    g.idx = d_idx;
    g.d2 = d_d2;
    g.counts = d_counts;
    g.err = d_err;
    g.est = est;
    g.packet_ctr = d_packet_ctr;
    g.chunk = chunk > 0 ? chunk : 1;
    g.fb_list = d_fb_list;
    g.stats = d_stats;
    g.fb_count = reinterpret_cast<unsigned long long*>(&d_fb->nq);
    const int sms = sm_count_k(device);
    const int bps = blocks_per_sm;
    if (single)
        e = (kmax <= 32) ? launch_group_seeded<1, 2>(g, sms, s, bps, d_head_kth, head_bytes, fp32)
                         : launch_group_seeded<2, 2>(g, sms, s, bps, d_head_kth, head_bytes, fp32);
    else
        e = (kmax <= 32) ? launch_group_seeded<1, 1>(g, sms, s, bps, d_head_kth, head_bytes, fp32)
                         : launch_group_seeded<2, 1>(g, sms, s, bps, d_head_kth, head_bytes, fp32);
    if (e != cudaSuccess) return e;
    // the queries handed back, exactly and without the provisional threshold
    return launch_knn_table(device, s, d_fb, single, 0, kmax, d_fb_list, bucket, d_idx, d_d2, d_counts, d_err,
                            bps, 0.0);
}

cudaError_t prepare_knn_dyn() {
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_knn<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)knn_smem<128>())) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_knn<256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)knn_smem<256>())) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_knn<512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)knn_smem<512>())) != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(k_knn<1024, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)knn_smem<1024>());
}

cudaError_t launch_knn(Cloud& c, const double* d_centers, uint64_t nq, uint32_t k, uint32_t* d_idx, double* d_d2,
                       uint32_t* d_counts) {
    if (nq == 0 || k == 0) return cudaSuccess;
    KnnArgs a{};
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
    a.bucket = c.packet ? c.knn_bucket : 0;  // the plain path descends to the leaves
    a.order = nullptr;
    if (c.packet) {  // curve-ordered queries: neighbouring warps share octants in cache
        cudaError_t e;
        if ((e = launch_query_order(c, d_centers, nq, &a.order)) != cudaSuccess) return e;
    }
    const uint64_t want = (nq + kKnnWarps - 1) / kKnnWarps;
    const uint64_t cap = (uint64_t)sm_count_k(c.device) * 16;
    const int grid = (int)(want < cap ? want : cap);
    if (c.packet && k <= 64) {
        // the FP32 filter (group kernel): centre-relative FP32 points, built on first use
        const bool f32 = fp32_on_knn(c.fp32_filter) && c.knn_packet != 0;
        if (f32 && !c.crel_built) {
            cudaError_t e;
            if ((e = launch_center_rel(c)) != cudaSuccess) return e;
            c.crel_built = true;
        }
        SearchReq r{};
        r.cv = cloud_view(c);
        r.centers = d_centers;
        r.q_begin = 0;
        r.q_end = nq;
        r.k = k;
        if (!c.knn_packet)
            return launch_knn_table(c.device, c.stream, nullptr, &r, nq, k, a.order, c.knn_bucket, d_idx, d_d2,
                                    d_counts, c.d_err.as<uint32_t>(), 0, c.knn_est);
        // groups of curve-ordered queries, then the exact per-query kernel for the queries they hand back
        cudaError_t e;
        if ((e = c.packet_ctr.reserve(256)) != cudaSuccess) return e;
        if ((e = c.knn_fb.reserve(16 + 4 * nq)) != cudaSuccess) return e;
        const uint64_t n_groups = (nq + kGrpQ - 1) / kGrpQ;
        const size_t head_bytes = 8 * (n_groups / kKnnHeadStride + 1);
        if ((e = c.knn_heads.reserve(head_bytes)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(c.packet_ctr.ptr, 0, 12, c.stream)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(c.knn_fb.ptr, 0, 8, c.stream)) != cudaSuccess) return e;
        KnnGroupArgs g{};
        g.single = r;
        g.grp = nullptr;
        g.packets = (nq + kGrpQ - 1) / kGrpQ;
        g.order = a.order;
        g.bucket = c.knn_bucket;
        g.idx = d_idx;
        g.d2 = d_d2;
        g.counts = d_counts;
        g.err = c.d_err.as<uint32_t>();
        g.est = c.knn_est;
        g.packet_ctr = c.packet_ctr.as<uint32_t>();
        g.chunk = c.knn_chunk;
        g.fb_count = c.knn_fb.as<unsigned long long>();
        g.fb_list = reinterpret_cast<uint32_t*>(c.knn_fb.as<unsigned char>() + 16);
        g.stats = f32 ? c.stats.as<unsigned long long>() + 2 : nullptr;  // oct_knn_filter_stats
        const int sms = sm_count_k(c.device);
        double* heads = c.knn_heads.as<double>();
        KernelClock clk(c, 1);
        e = (k <= 32) ? launch_group_seeded<1, 0>(g, sms, c.stream, 0, heads, head_bytes, f32)
                      : launch_group_seeded<2, 0>(g, sms, c.stream, 0, heads, head_bytes, f32);
        clk.stop();
        if (e != cudaSuccess) return e;
        KnnTableArgs f{};
        f.single = r;
        f.nq = nq;
        f.nq_dev = g.fb_count;
        f.order = g.fb_list;
        f.bucket = c.knn_bucket;
        f.idx = d_idx;
        f.d2 = d_d2;
        f.counts = d_counts;
        f.err = g.err;
        f.est = 0.0;  // exact without the provisional threshold
        const int fgrid = sms * 16;
        if (k <= 32) k_knn_reg<1, 0><<<fgrid, kKnnThreads, 0, c.stream>>>(f);
        else k_knn_reg<2, 0><<<fgrid, kKnnThreads, 0, c.stream>>>(f);
        return cudaGetLastError();
    }
    if (k <= 32) return launch_l<32>(a, grid, c.stream, c.packet != 0);
    if (k <= 64) return launch_l<64>(a, grid, c.stream, c.packet != 0);
    if (k <= 128) return launch_l<128>(a, grid, c.stream, c.packet != 0);
    if (k <= 256) return launch_l<256>(a, grid, c.stream, c.packet != 0);
    if (k <= 512) return launch_l<512>(a, grid, c.stream, c.packet != 0);
    return launch_l<1024>(a, grid, c.stream, c.packet != 0);
}

// A kernel of this file's device code, for preload_kernels.
const void* kernel_anchor_knn_search() { return reinterpret_cast<const void*>(&k_knn_reg<2, 0>); }

}  // namespace octb
