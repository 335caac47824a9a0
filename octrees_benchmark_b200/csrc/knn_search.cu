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
    }
    const uint64_t nwarps = (uint64_t)gridDim.x * kKnnWarps;
    for (uint64_t w = (uint64_t)blockIdx.x * kKnnWarps + warp; w < nq; w += nwarps) {
        const uint64_t qpos = q0 + w;
        uint32_t ri = 0;
        if (MULTI) {  // the request whose positions contain qpos (q_begin ascending)
            uint32_t lo = 0, hi = nreq;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (reqs[mid].q_begin <= qpos) lo = mid;
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
        const uint64_t q = a.order ? a.order[qpos] : qpos;  // global query position
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
// Packet kNN: 32 curve-ordered queries per warp, one per lane.
//
// The warp walks the tree once for its 32 queries.  Every lane keeps its own
// k best (squared distance, index) pairs in a max-heap in shared memory (root =
// the current k-th pair), so a lane's threshold is the root once the heap is
// full.  A node is visited by the lanes whose lower bound to it (the
// reference's clamp-to-box distance) does not exceed their threshold; the
// children of a node are pushed with the mask of lanes that accept them,
// nearest to the packet's centroid on top.  A leaf's points are staged in
// shared memory once per warp and every visiting lane offers them to its heap.
// At the end each lane heap-sorts its pairs into ascending (distance, index)
// order, which is the device's tie rule.
// ---------------------------------------------------------------------------

template <int KCAP>
struct KnnPkShape {
    static constexpr int kWarps = (KCAP <= 64) ? 4 : 2;
};

__device__ __forceinline__ bool pair_gt(double da, uint32_t ia, double db, uint32_t ib) {
    return (da > db) || (da == db && ia > ib);
}

template <int KCAP>
__global__ void __launch_bounds__(32 * KnnPkShape<KCAP>::kWarps) k_knn_packet(KnnArgs a, const uint32_t* order,
                                                                              uint32_t* packet_ctr) {
    constexpr int W = KnnPkShape<KCAP>::kWarps;
    extern __shared__ __align__(16) unsigned char smem[];
    // per warp: heap distances [KCAP][32], heap indices [KCAP][32]
    double* hd_all = reinterpret_cast<double*>(smem);
    uint32_t* hi_all = reinterpret_cast<uint32_t*>(hd_all + (size_t)W * KCAP * 32);
    __shared__ uint32_t st_node[W][kKnnStack];
    __shared__ uint32_t st_mask[W][kKnnStack];
    __shared__ uint8_t st_depth[W][kKnnStack];
    __shared__ double sx[W][32], sy[W][32], sz[W][32];
    __shared__ double s_radii[kMaxDepth + 1][3];
    for (int i = threadIdx.x; i < (kMaxDepth + 1) * 3; i += 32 * W) (&s_radii[0][0])[i] = (&a.geom->radii[0][0])[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lbit = 1u << lane;
    double* hd = hd_all + (size_t)warp * KCAP * 32;
    uint32_t* hx = hi_all + (size_t)warp * KCAP * 32;
#define HD(j) hd[(j) * 32 + lane]
#define HX(j) hx[(j) * 32 + lane]
    const uint32_t K = a.k;

    for (;;) {
        uint32_t packet = 0;
        if (lane == 0) packet = atomicAdd(packet_ctr, 1u);
        packet = __shfl_sync(0xffffffffu, packet, 0);
        const uint64_t i0 = (uint64_t)packet * 32;
        if (i0 >= a.nq) break;
        const uint64_t qpos = i0 + lane;
        const bool valid = qpos < a.nq;
        const uint32_t qi = valid ? order[qpos] : 0u;
        const double p[3] = {a.q[3ull * qi], a.q[3ull * qi + 1], a.q[3ull * qi + 2]};
        // packet centroid, used only to order children
        const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
        const double inv = 1.0 / (double)__popc(vmask);
        double cen[3];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            double v = valid ? p[ax] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            cen[ax] = v * inv;
        }
        uint32_t hs = 0;  // heap size of this lane
        auto thr_d = [&]() { return (hs < K) ? (double)INFINITY : HD(0); };
        auto offer = [&](double d, uint32_t idx) {
            if (hs < K) {
                uint32_t j = hs++;
                while (j > 0) {
                    const uint32_t pj = (j - 1) >> 1;
                    if (!pair_gt(d, idx, HD(pj), HX(pj))) break;
                    HD(j) = HD(pj);
                    HX(j) = HX(pj);
                    j = pj;
                }
                HD(j) = d;
                HX(j) = idx;
            } else if (pair_less(d, idx, HD(0), HX(0))) {
                uint32_t j = 0;
                for (;;) {
                    const uint32_t l = 2 * j + 1;
                    if (l >= K) break;
                    uint32_t m = l;
                    if (l + 1 < K && pair_gt(HD(l + 1), HX(l + 1), HD(l), HX(l))) m = l + 1;
                    if (!pair_gt(HD(m), HX(m), d, idx)) break;
                    HD(j) = HD(m);
                    HX(j) = HX(m);
                    j = m;
                }
                HD(j) = d;
                HX(j) = idx;
            }
        };

        int sp = 0;
        if (lane == 0) {
            st_node[warp][0] = 0;
            st_mask[warp][0] = vmask;
            st_depth[warp][0] = 0;
        }
        __syncwarp();
        if (vmask) sp = 1;
        bool failed = false;
        while (sp > 0) {
            --sp;
            const uint32_t node = st_node[warp][sp];
            const uint32_t mask = st_mask[warp][sp];
            const uint32_t depth = st_depth[warp][sp];
            __syncwarp();
            // lanes still interested: lower bound within their threshold (root: bound 0)
            bool act = (mask & lbit) != 0;
            if (act && depth > 0) act = !(dist_po(p, a.centers + 3ull * node, s_radii[depth]) > thr_d());
            const uint32_t am = __ballot_sync(0xffffffffu, act);
            if (!am) continue;
            const uint32_t fc = a.offsets[node];
            if (fc == 0) {
                const uint2 rg = a.ranges[node];
                for (uint32_t b = rg.x; b < rg.y; b += 32) {
                    const uint32_t idx = b + lane;
                    if (idx < rg.y) {
                        sx[warp][lane] = a.xs[idx];
                        sy[warp][lane] = a.ys[idx];
                        sz[warp][lane] = a.zs[idx];
                    }
                    __syncwarp();
                    const uint32_t m = (rg.y - b < 32u) ? (rg.y - b) : 32u;
                    if (act) {
                        for (uint32_t t = 0; t < m; ++t) {
                            const double d = dist_pp(p[0], p[1], p[2], sx[warp][t], sy[warp][t], sz[warp][t]);
                            if (hs < K || !pair_gt(d, b + t, HD(0), HX(0))) offer(d, b + t);
                        }
                    }
                    __syncwarp();
                }
                continue;
            }
            const uint32_t cd = depth + 1;
            uint32_t cm[8];
            const double th = act ? thr_d() : -1.0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                bool ok = false;
                if (act) ok = !(dist_po(p, a.centers + 3ull * (fc + j), s_radii[cd]) > th);
                cm[j] = __ballot_sync(0xffffffffu, ok);
            }
            // order key: the centroid's bound to each child, computed on lanes 0..7
            double key = INFINITY;
            if (lane < 8) key = dist_po(cen, a.centers + 3ull * (fc + lane), s_radii[cd]);
            int np = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) np += (cm[j] != 0);
            if (sp + np > kKnnStack) {
                failed = true;
                break;
            }
            // slot of child j among pushed children: farther (or equal and higher octant) ones go deeper
            int pos = 0;
            uint32_t myc = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const double kj = __shfl_sync(0xffffffffu, key, j);
                if (lane < 8 && cm[j] != 0 && j != lane && ((kj > key) || (kj == key && j > lane))) ++pos;
                if (lane == j) myc = cm[j];
            }
            if (lane < 8 && myc != 0) {
                st_node[warp][sp + pos] = fc + lane;
                st_mask[warp][sp + pos] = myc;
                st_depth[warp][sp + pos] = (uint8_t)cd;
            }
            __syncwarp();
            sp += np;
        }
        if (failed) set_err(a.err, kErrStackOverflow);
        if (valid) {
            // heap-sort into ascending (distance, index)
            for (uint32_t e = hs; e > 1; --e) {
                const uint32_t last = e - 1;
                const double d = HD(last);
                const uint32_t ix = HX(last);
                HD(last) = HD(0);
                HX(last) = HX(0);
                uint32_t j = 0;
                for (;;) {
                    const uint32_t l = 2 * j + 1;
                    if (l >= last) break;
                    uint32_t m = l;
                    if (l + 1 < last && pair_gt(HD(l + 1), HX(l + 1), HD(l), HX(l))) m = l + 1;
                    if (!pair_gt(HD(m), HX(m), d, ix)) break;
                    HD(j) = HD(m);
                    HX(j) = HX(m);
                    j = m;
                }
                HD(j) = d;
                HX(j) = ix;
            }
            const uint64_t o = (uint64_t)qi * K;
            for (uint32_t j = 0; j < K; ++j) {
                a.idx[o + j] = (j < hs) ? HX(j) : 0xffffffffu;
                a.d2[o + j] = (j < hs) ? HD(j) : (double)INFINITY;
            }
            if (a.counts) a.counts[qi] = hs;
        }
        __syncwarp();
    }
#undef HD
#undef HX
}

template <int KCAP>
cudaError_t launch_knn_pk(const KnnArgs& a, const uint32_t* order, uint32_t* ctr, int sms, cudaStream_t s) {
    constexpr int W = KnnPkShape<KCAP>::kWarps;
    const size_t smem = (size_t)W * KCAP * 32 * 12;
    cudaError_t e = cudaFuncSetAttribute(k_knn_packet<KCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint64_t packets = (a.nq + 31) / 32;
    const uint64_t want = (packets + W - 1) / W;
    const uint64_t cap = (uint64_t)sms * 8;
    const int grid = (int)(want < cap ? want : cap);
    k_knn_packet<KCAP><<<grid, 32 * W, smem, s>>>(a, order, ctr);
    return cudaGetLastError();
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
    KnnTableArgs a;
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
    if (c.packet && c.knn_packet && k <= 128) {
        cudaError_t e;
        const uint32_t* order = a.order;
        if ((e = c.packet_ctr.reserve(256)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(c.packet_ctr.ptr, 0, 4, c.stream)) != cudaSuccess) return e;
        uint32_t* ctr = c.packet_ctr.as<uint32_t>();
        const int sms = sm_count_k(c.device);
        if (k <= 16) return launch_knn_pk<16>(a, order, ctr, sms, c.stream);
        if (k <= 32) return launch_knn_pk<32>(a, order, ctr, sms, c.stream);
        if (k <= 64) return launch_knn_pk<64>(a, order, ctr, sms, c.stream);
        return launch_knn_pk<128>(a, order, ctr, sms, c.stream);
    }
    const uint64_t want = (nq + kKnnWarps - 1) / kKnnWarps;
    const uint64_t cap = (uint64_t)sm_count_k(c.device) * 16;
    const int grid = (int)(want < cap ? want : cap);
    if (c.packet && k <= 64) {
        SearchReq r{};
        r.cv = cloud_view(c);
        r.centers = d_centers;
        r.q_begin = 0;
        r.q_end = nq;
        r.k = k;
        return launch_knn_table(c.device, c.stream, nullptr, &r, nq, k, a.order, c.knn_bucket, d_idx, d_d2, d_counts,
                                c.d_err.as<uint32_t>(), 0, c.knn_est);
    }
    if (k <= 32) return launch_l<32>(a, grid, c.stream, c.packet != 0);
    if (k <= 64) return launch_l<64>(a, grid, c.stream, c.packet != 0);
    if (k <= 128) return launch_l<128>(a, grid, c.stream, c.packet != 0);
    if (k <= 256) return launch_l<256>(a, grid, c.stream, c.packet != 0);
    if (k <= 512) return launch_l<512>(a, grid, c.stream, c.packet != 0);
    return launch_l<1024>(a, grid, c.stream, c.packet != 0);
}

}  // namespace octb
