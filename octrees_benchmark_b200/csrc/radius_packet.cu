// Batched ("packet") radius search: neighbors / neighborsPrune / neighborsStruct
// for 32 spatially ordered queries per warp.
//
// Reference path replaced: the same as radius_search.cu - singleTraversal
// (inc/structures/linear_octree.hpp:653-686) with the criteria and leaf actions of
// neighborsStruct (695-736), neighborsPrune (746-784) and neighbors (796-816).
//
// B200 design.  The query centres are first ordered along the cloud's curve
// (launch_query_order), so the 32 queries of a warp are neighbours in space and
// need almost the same octants.  The warp walks the tree once for all of them:
// at every internal node each lane judges the 8 children for its own query (the
// reference's predicates, bit for bit), and a child is pushed with two lane
// masks - the lanes for which it is fully inside (they emit its whole range
// when it is popped) and the lanes that must descend into it.  Pushing the
// children lowest octant last keeps every lane's output in ascending order.
// Leaves, FP64 neighbors / neighborsPrune (the transposed test): the lanes load
// 32 consecutive points and test them against one query of the descend mask at
// a time, so all lanes work and the ballot is that query's hit mask, stored in
// one coalesced write.  neighborsStruct and the FP32 form stage a leaf's points
// in shared memory and every lane of the mask tests its own query against all
// of them.  Fully-inside ranges are written by the whole warp.  Packets are
// handed out by an atomic counter so that long and short packets balance.
//
// Output: count pass + scan + fill at the scanned offsets, or one pass in which
// every query appends its results to its own chain of 64-entry chunks (see
// k_radius_packet's CHUNK form) that k_chunk_compact moves into the CSR array.
//
// FP32 variant (the precision form): each sorted point also has FP32
// coordinates relative to its leaf's centre (x, y, z computed in FP64 and
// rounded once; w = their L1 norm).  A lane tests its query, made relative to
// the same centre, in FP32; a point whose FP32 result lies within a rigorous
// error band of the decision boundary is re-tested in FP64 on the original
// coordinates with the reference's expression, so every decision is still the
// reference's.  Band (sphere / circle, inside iff d2 < r2 / d2 <= r2):
//   |d2_fp32 - d2| <= 2^-23 (|q|_1 + |p|_1 + 1.74 r) r + 3 2^-24 d2 near the
//   boundary, plus 2^-24 r2 for rounding r2 to FP32; the band used is 2 to 4
//   times that:  2^-21 ((|q|_1 + |p|_1 + 2 r) r + r2).
// Cube / square: per axis, the interval bounds bmin = c - r and bmax = c + r
// (FP64) are made leaf-relative and rounded to FP32; an axis is certain when
// its margin exceeds 2^-22 (|p_i| + |bound_i|).
#include <cfloat>

#include "cloud.h"
#include "search_kernels.cuh"

namespace octb {

namespace {

constexpr int kPkWarps = 4;
constexpr int kPkThreads = 32 * kPkWarps;
constexpr int kPkStack = 8 * (kMaxDepth + 1);
constexpr uint32_t kChunk = kResultChunk;  // entries per result chunk (one-pass mode)
constexpr uint32_t kNoChunk = 0xffffffffu;

struct PacketArgs {
    SearchReq single;           // the request of a single-cloud search (grp == null); with
                                // one_cloud, single.cv is the cloud of every request of grp
    const DynGroup* grp;        // sizes and request table of a batch group (device)
    uint64_t packets;           // packets of a single-request launch
    bool one_cloud;             // host dispatch: grp's requests all search single.cv
    const uint32_t* order;      // query visiting order (global positions), or null
    unsigned long long* counts;
    unsigned long long* counts2;
    const unsigned long long* offs;
    uint32_t* out;
    uint64_t out_cap;
    uint32_t* packet_ctr;
    unsigned long long* stats;  // [0] point tests, [1] FP64 re-tests
    uint32_t* err;
    // one-pass mode: each query's results go to its own chain of kChunk-entry chunks
    uint32_t* chunk_pool;       // chunk_cap x kChunk entries
    uint32_t* chunk_next;       // next chunk of a chain (chunk_cap)
    uint32_t* chunk_first;      // first chunk of each query (per query position)
    uint32_t* chunk_ctr;        // chunks handed out
    uint32_t chunk_cap;
};

// Per-lane FP32 context of one leaf.
struct LeafCtx {
    float qx, qy, qz;  // query centre relative to the leaf centre
    float r2f;         // radius^2 rounded to FP32 (sphere, circle)
    float b0, b1;      // band = b0 + b1 * |p|_1 (sphere, circle)
    float lo[3], hi[3], tlo[3], thi[3];  // relative interval bounds and their tolerances (cube, square)
};

template <int KT>
__device__ __forceinline__ void leaf_ctx(const SearchKernel& k, const double* lc, LeafCtx& c) {
    c.qx = (float)dsub(k.c[0], lc[0]);
    c.qy = (float)dsub(k.c[1], lc[1]);
    c.qz = (float)dsub(k.c[2], lc[2]);
    const float r = (float)k.r;
    if constexpr (KT == kSphere || KT == kCircle) {
        const float q1 = fabsf(c.qx) + fabsf(c.qy) + ((KT == kSphere) ? fabsf(c.qz) : 0.0f);
        c.r2f = (float)k.r2;
        const float s = 4.76837158203125e-07f;  // 2^-21
        c.b0 = s * ((q1 + 2.0f * r) * r + c.r2f) + FLT_MIN;
        c.b1 = s * r;
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            c.lo[a] = (float)dsub(k.bmin[a], lc[a]);
            c.hi[a] = (float)dsub(k.bmax[a], lc[a]);
            c.tlo[a] = 2.384185791015625e-07f * fabsf(c.lo[a]);  // 2^-22 |bound|
            c.thi[a] = 2.384185791015625e-07f * fabsf(c.hi[a]);
        }
    }
}

// FP32 test: 1 inside, 0 outside, -1 undecided (re-test in FP64).
template <int KT>
__device__ __forceinline__ int f32_test(const LeafCtx& c, float4 p) {
    if constexpr (KT == kSphere || KT == kCircle) {
        const float dx = p.x - c.qx, dy = p.y - c.qy;
        float d2 = __fmaf_rn(dy, dy, __fmul_rn(dx, dx));
        if constexpr (KT == kSphere) {
            const float dz = p.z - c.qz;
            d2 = __fmaf_rn(dz, dz, d2);
        }
        const float band = __fmaf_rn(c.b1, p.w, c.b0);
        if (d2 < c.r2f - band) return 1;
        if (d2 > c.r2f + band) return 0;
        return -1;
    } else {
        constexpr int D = (KT == kCube) ? 3 : 2;
        const float pv[3] = {p.x, p.y, p.z};
        const float tp = 2.384185791015625e-07f * p.w;  // 2^-22 |p|_1 >= 2^-22 |p_i|
        bool sure_in = true;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            const float ml = pv[a] - c.lo[a], mh = c.hi[a] - pv[a];
            const float tl = tp + c.tlo[a], th = tp + c.thi[a];
            if (ml < -tl || mh < -th) return 0;
            sure_in = sure_in && (ml > tl) && (mh > th);
        }
        return sure_in ? 1 : -1;
    }
}

// MULTI 0: one request, read from the kernel parameters (constant-bank
// operands, no registers held).  1: a request table; the cloud pointers of the
// warp's current request live in shared memory (RQV), so the hot loops do not
// re-load them from the table.  2: a request table whose requests are all on
// one cloud, whose pointers are kernel parameters again (no shared-memory
// reads in the hot loops).
#define RQ(f) (MULTI ? reqs[cur_req].f : a.single.f)
#define RQV(f) (MULTI == 1 ? s_view[warp].f : a.single.cv.f)

// Query parameters of lane j for the transposed leaf and child tests, one
// 48-byte row per query so that a test reads them with 16-byte loads: sphere /
// circle (c0, c1, c2, r2, r, -), cube / square (bmin0..2, bmax0..2).
constexpr int kQpRow = 6;
__device__ __forceinline__ double2 ld_d2(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ float4 ld_f4(const float* p) { return *reinterpret_cast<const float4*>(p); }

template <int KT>
__device__ __forceinline__ void put_query(double (*q)[kQpRow], int lane, const SearchKernel& k) {
    if constexpr (KT == kSphere || KT == kCircle) {
        q[lane][0] = k.c[0];
        q[lane][1] = k.c[1];
        q[lane][2] = k.c[2];
        q[lane][3] = k.r2;
        q[lane][4] = k.r;
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            q[lane][a] = k.bmin[a];
            q[lane][3 + a] = k.bmax[a];
        }
    }
}

// Lane j's SearchKernel back from put_query's copy: the fields the box tests,
// the leaf tests and the FP32 context read (bounds of a sphere / circle are
// recomputed by init's own expressions, so they are the same values).
template <int KT>
__device__ __forceinline__ SearchKernel kernel_of(const double (*q)[kQpRow], int j) {
    SearchKernel k;
    if constexpr (KT == kSphere || KT == kCircle) {
        const double2 a = ld_d2(&q[j][0]), b = ld_d2(&q[j][2]);
        k.c[0] = a.x;
        k.c[1] = a.y;
        k.c[2] = b.x;
        k.r2 = b.y;
        k.r = q[j][4];
#pragma unroll
        for (int a2 = 0; a2 < 3; ++a2) {
            k.bmin[a2] = dsub(k.c[a2], k.r);
            k.bmax[a2] = dadd(k.c[a2], k.r);
        }
    } else {  // cube / square tests read the bounds only
        const double2 a = ld_d2(&q[j][0]), b = ld_d2(&q[j][2]), c = ld_d2(&q[j][4]);
        k.r = k.r2 = 0.0;
        k.c[0] = k.c[1] = k.c[2] = 0.0;
        k.bmin[0] = a.x;
        k.bmin[1] = a.y;
        k.bmin[2] = b.x;
        k.bmax[0] = b.y;
        k.bmax[1] = c.x;
        k.bmax[2] = c.y;
    }
    return k;
}

// FP32 leaf context of lane j's query for the transposed FP32 test, one row
// per query: sphere / circle (qx, qy, qz, r2f | b0, b1, -, -), cube / square
// (lo0..2, hi0 | hi1, hi2, tlo0, tlo1 | tlo2, thi0..2).
template <int KT>
__device__ __forceinline__ void put_ctx(float* row, const LeafCtx& c) {
    if constexpr (KT == kSphere || KT == kCircle) {
        row[0] = c.qx;
        row[1] = c.qy;
        row[2] = c.qz;
        row[3] = c.r2f;
        row[4] = c.b0;
        row[5] = c.b1;
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            row[a] = c.lo[a];
            row[3 + a] = c.hi[a];
            row[6 + a] = c.tlo[a];
            row[9 + a] = c.thi[a];
        }
    }
}
template <int KT>
__device__ __forceinline__ LeafCtx get_ctx(const float* row) {
    LeafCtx c;
    if constexpr (KT == kSphere || KT == kCircle) {
        const float4 a = ld_f4(row);
        const float2 b = *reinterpret_cast<const float2*>(row + 4);
        c.qx = a.x;
        c.qy = a.y;
        c.qz = a.z;
        c.r2f = a.w;
        c.b0 = b.x;
        c.b1 = b.y;
    } else {
        const float4 a = ld_f4(row), b = ld_f4(row + 4), d = ld_f4(row + 8);
        c.lo[0] = a.x;
        c.lo[1] = a.y;
        c.lo[2] = a.z;
        c.hi[0] = a.w;
        c.hi[1] = b.x;
        c.hi[2] = b.y;
        c.tlo[0] = b.z;
        c.tlo[1] = b.w;
        c.tlo[2] = d.x;
        c.thi[0] = d.y;
        c.thi[1] = d.z;
        c.thi[2] = d.w;
    }
    return c;
}

// is_inside of lane j's query for point p: the same expressions, operand for operand.
template <int KT>
__device__ __forceinline__ bool inside_of(const double (*q)[kQpRow], int j, double px, double py, double pz) {
    if constexpr (KT == kSphere) {
        const double2 a = ld_d2(&q[j][0]), b = ld_d2(&q[j][2]);
        return dsq3(dsub(px, a.x), dsub(py, a.y), dsub(pz, b.x)) < b.y;
    } else if constexpr (KT == kCircle) {
        const double2 a = ld_d2(&q[j][0]), b = ld_d2(&q[j][2]);
        return dsq2(dsub(px, a.x), dsub(py, a.y)) <= b.y;
    } else {
        const double2 a = ld_d2(&q[j][0]), b = ld_d2(&q[j][2]), c = ld_d2(&q[j][4]);
        // bmin = (a.x, a.y, b.x), bmax = (b.y, c.x, c.y)
        if constexpr (KT == kCube)
            return px >= a.x && px <= b.y && py >= a.y && py <= c.x && pz >= b.x && pz <= c.y;
        else
            return px >= a.x && px <= b.y && py >= a.y && py <= c.x;
    }
}

// CHUNK (with FILL, transposed form only): one pass instead of count + fill.
// Each query appends its results to its own chain of kChunk-entry chunks taken
// from a pool (contiguous chunks for one long range, so positions stay
// linear); per query the count and the first chunk are written, and
// k_chunk_compact moves every chain into the CSR array after the scan.
template <int KT, int ALGO, bool FILL, bool F32, int MULTI, bool CHUNK = false>
__global__ void __launch_bounds__(kPkThreads) k_radius_packet(PacketArgs a) {
    // Transposed leaf test (neighbors / neighborsPrune, FP64 or FP32 filter): the
    // lanes hold consecutive points and test them against one query of the mask
    // at a time, so every lane does useful work and the ballot is that query's
    // hit mask.  The FP32 form reads the points' leaf-relative coordinates and
    // each query's context for the leaf (made once per leaf by the query's own
    // lane); a point inside the error band is re-tested in FP64.
    constexpr bool kT = (ALGO != kStruct);
    static_assert(!CHUNK || (FILL && kT), "one-pass mode needs the transposed form");
    constexpr int kStage = (kT || F32) ? 1 : kPkWarps;  // FP64 point staging, per-lane FP64 form only
    constexpr int kCtxF = (KT == kSphere || KT == kCircle) ? 8 : 12;  // floats of a query's FP32 leaf context row
    __shared__ __align__(16) float s_ctx[(F32 && kT) ? kPkWarps : 1][32][kCtxF];
    __shared__ CloudView s_view[MULTI == 1 ? kPkWarps : 1];
    __shared__ uint32_t st_node[kPkWarps][kPkStack];
    __shared__ uint32_t st_fc[kPkWarps][kPkStack];     // first child, 0 for a leaf
    __shared__ uint2 st_rg[kPkWarps][kPkStack];        // point range
    __shared__ uint32_t st_over[kPkWarps][kPkStack];
    __shared__ uint32_t st_in[kPkWarps][kPkStack];
    __shared__ uint8_t st_depth[kPkWarps][kPkStack];
    __shared__ double s_rad[kPkWarps][kMaxDepth + 1][3];
    __shared__ __align__(16) double s_qp[kPkWarps][32][kQpRow];
    __shared__ double sx[kStage][32], sy[kStage][32], sz[kStage][32];
    __shared__ float4 sp[(F32 && !kT) ? kPkWarps : 1][32];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double (*s_radii)[3] = s_rad[warp];
    uint32_t cur_cloud = 0xffffffffu;
    uint32_t cur_req = 0;
    const SearchReq* reqs = nullptr;
    uint32_t nreq = 1;
    uint64_t packets = a.packets;
    if (MULTI) {
        reqs = a.grp->reqs;
        nreq = a.grp->nreq;
        packets = a.grp->packets;
    }
    const uint32_t lbit = 1u << lane;
    uint32_t* sn = st_node[warp];
    uint32_t* sf = st_fc[warp];
    uint2* sr = st_rg[warp];
    uint32_t* so = st_over[warp];
    uint32_t* si = st_in[warp];
    uint8_t* sd = st_depth[warp];
    unsigned long long n_tests = 0, n_retests = 0;

    for (;;) {
        uint32_t packet = 0;
        if (lane == 0) packet = atomicAdd(a.packet_ctr, 1u);
        packet = __shfl_sync(0xffffffffu, packet, 0);
        if (packet >= packets) break;
        // the request of this packet: packet_begin is ascending over the table
        if (MULTI) {
            uint32_t lo = 0, hi = nreq;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (reqs[mid].packet_begin <= packet) lo = mid;
                else hi = mid;
            }
            cur_req = lo;
        }
        if (RQ(cloud_id) != cur_cloud) {  // this warp's level radii and cloud follow the packet's cloud
            __syncwarp();
            const double* gr = &RQ(cv.geom)->radii[0][0];
            for (int t = lane; t < (kMaxDepth + 1) * 3; t += 32) (&s_radii[0][0])[t] = gr[t];
            if (MULTI == 1 && lane == 0) s_view[warp] = reqs[cur_req].cv;
            cur_cloud = RQ(cloud_id);
            __syncwarp();
        }
        const uint64_t q_begin = RQ(q_begin);
        const uint64_t i = q_begin + 32ull * (packet - RQ(packet_begin)) + lane;
        const bool valid = i < RQ(q_end);
        const uint64_t qg = valid ? (a.order ? (uint64_t)a.order[i] : i) : q_begin;  // global query position
        const uint64_t ql = qg - q_begin;                                              // within the request
        const uint32_t qi = (uint32_t)qg;
        const double* qc = RQ(centers);
        const double* qrad = RQ(radii);
        const uint32_t approx_cut = (ALGO == kStruct) ? RQ(approx_cut) : 0u;
        const bool approx_upper = (ALGO == kStruct) && RQ(approx_upper) != 0;
        SearchKernel k;
        k.init(qc[3 * ql], qc[3 * ql + 1], qc[3 * ql + 2], qrad ? qrad[ql] : RQ(radius));
        __syncwarp();  // the previous packet's reads of s_qp are done
        put_query<KT>(s_qp[warp], lane, k);  // read by the other lanes after a __syncwarp
        unsigned long long cnt = 0, cnt2 = 0, base = 0;
        if (FILL && !CHUNK && valid) base = a.offs[qi];
        bool overflow = false;
        bool open = false;  // neighborsStruct: a run of inside points is open
        uint32_t rs = 0;
        // one-pass mode: this lane's chain (current chunk, entries used in it, first chunk)
        uint32_t ck_cur = kNoChunk, ck_fill = kChunk, ck_first = kNoChunk;
        bool ck_over = false;

        // Reserve n > 0 entries at the end of lane j's chain (warp-uniform call):
        // returns where they go - the first `room` continue chunk `cur`, the rest
        // are linear from chunk `nc` on (new chunks taken as one contiguous run).
        struct ChunkPos {
            uint32_t cur, fill, room, nc;
        };
        auto chunk_reserve = [&](int j, uint32_t n) -> ChunkPos {
            ChunkPos p;
            p.cur = __shfl_sync(0xffffffffu, ck_cur, j);
            p.fill = __shfl_sync(0xffffffffu, ck_fill, j);
            p.room = kChunk - p.fill;
            p.nc = kNoChunk;
            if (n > p.room) {
                const uint32_t m = (n - p.room + kChunk - 1) / kChunk;
                uint32_t nc = 0;
                if (lane == 0) nc = atomicAdd(a.chunk_ctr, m);
                nc = __shfl_sync(0xffffffffu, nc, 0);
                p.nc = nc;
                const bool fits = (uint64_t)nc + m <= a.chunk_cap;
                if (!fits) ck_over = true;  // the pool is too small: counts stay exact, the host re-runs
                if (fits) {
                    if (lane == 0 && p.cur != kNoChunk) a.chunk_next[p.cur] = nc;
                    for (uint32_t t = lane; t + 1 < m; t += 32) a.chunk_next[nc + t] = nc + t + 1;
                }
                if (lane == j) {
                    if (ck_cur == kNoChunk) ck_first = nc;
                    ck_cur = nc + m - 1;
                    ck_fill = n - p.room - (m - 1) * kChunk;
                }
            } else if (lane == j) {
                ck_fill += n;
            }
            if (lane == j) cnt += n;
            return p;
        };
        auto chunk_store = [&](const ChunkPos& p, uint32_t r, uint32_t v) {
            const uint64_t pos = (r < p.room) ? (uint64_t)p.cur * kChunk + p.fill + r
                                              : (uint64_t)p.nc * kChunk + (r - p.room);
            if (pos < (uint64_t)a.chunk_cap * kChunk) a.chunk_pool[pos] = v;
        };

        auto emit_range = [&](uint32_t f, uint32_t l) {  // per lane
            if constexpr (ALGO == kStruct) {
                if (FILL) {
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
                    for (uint32_t t = f; t < l; ++t) {
                        const unsigned long long o = base + cnt + (t - f);
                        if (o < a.out_cap) a.out[o] = t;
                        else overflow = true;
                    }
                }
                cnt += (unsigned long long)(l - f);
            }
        };
        auto hit = [&](uint32_t idx, bool in) {  // per lane, points in order
            if constexpr (ALGO == kStruct) {
                if (in && !open) {
                    open = true;
                    rs = idx;
                } else if (!in && open) {
                    open = false;
                    emit_range(rs, idx);
                }
            } else {
                if (in) {
                    if (FILL) {
                        const unsigned long long o = base + cnt;
                        if (o < a.out_cap) a.out[o] = idx;
                        else overflow = true;
                    }
                    ++cnt;
                }
            }
        };
        auto scan_leaf = [&](uint32_t node, uint2 rg, uint32_t mask) {
            if constexpr (kT) {
                if constexpr (F32) {  // each query of the mask: its context for this leaf, from its own lane
                    __syncwarp();
                    if ((mask >> lane) & 1u) {
                        LeafCtx ctx;
                        leaf_ctx<KT>(kernel_of<KT>(s_qp[warp], lane), RQV(centers) + 3ull * node, ctx);
                        put_ctx<KT>(s_ctx[warp][lane], ctx);
                    }
                    __syncwarp();
                } else {
                    (void)node;
                }
                for (uint32_t b = rg.x; b < rg.y; b += 32) {
                    const uint32_t idx = b + lane;
                    const bool in_range = idx < rg.y;
                    double px = 0.0, py = 0.0, pz = 0.0;
                    float4 pf = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    if (in_range) {
                        if constexpr (F32) {
                            pf = RQV(rel)[idx];
                        } else {
                            px = RQV(xs)[idx];
                            py = RQV(ys)[idx];
                            pz = RQV(zs)[idx];
                        }
                    }
                    // query j's hits among the lanes' points: appended to its chunks, or stored ascending
                    // in one coalesced store (FILL), and counted
                    auto take = [&](int j, bool in) {
                        const uint32_t hb = __ballot_sync(0xffffffffu, in);
                        if constexpr (CHUNK) {
                            if (hb) {
                                const ChunkPos p = chunk_reserve(j, __popc(hb));
                                if (in) chunk_store(p, __popc(hb & lanemask_lt()), idx);
                            }
                            return;
                        }
                        if (FILL && hb) {
                            const unsigned long long o0 = __shfl_sync(0xffffffffu, base + cnt, j);
                            if (in) {
                                const unsigned long long o = o0 + __popc(hb & lanemask_lt());
                                if (o < a.out_cap) a.out[o] = idx;
                                else overflow = true;
                            }
                        }
                        if (lane == j) cnt += __popc(hb);
                    };
                    uint32_t rem = mask;
                    while (rem) {
                        const int j = __ffs(rem) - 1;
                        rem &= rem - 1;
                        if constexpr (F32) {
                            bool in;
                            const int r = in_range ? f32_test<KT>(get_ctx<KT>(s_ctx[warp][j]), pf) : 0;
                            if (r < 0) {  // inside the error band: the reference's FP64 expression decides
                                in = inside_of<KT>(s_qp[warp], j, RQV(xs)[idx], RQV(ys)[idx], RQV(zs)[idx]);
                                ++n_retests;
                            } else {
                                in = r > 0;
                            }
                            take(j, in);
                        } else {
                            // two queries at a time: their FP64 tests are independent, so their latencies
                            // overlap instead of adding up
                            const bool two = rem != 0;
                            const int j2 = two ? __ffs(rem) - 1 : j;
                            if (two) rem &= rem - 1;
                            const bool in = in_range && inside_of<KT>(s_qp[warp], j, px, py, pz);
                            const bool in2 = two && in_range && inside_of<KT>(s_qp[warp], j2, px, py, pz);
                            take(j, in);
                            if (two) take(j2, in2);
                        }
                    }
                    if (lane == 0) n_tests += (unsigned long long)__popc(mask) * ((rg.y - b < 32u) ? (rg.y - b) : 32u);
                }
            } else {
            const bool mine = (mask & lbit) != 0;
            LeafCtx ctx;
            if (F32 && mine) leaf_ctx<KT>(k, RQV(centers) + 3ull * node, ctx);
            for (uint32_t b = rg.x; b < rg.y; b += 32) {
                const uint32_t idx = b + lane;
                if (idx < rg.y) {
                    if constexpr (F32) {
                        sp[warp][lane] = RQV(rel)[idx];
                    } else {
                        sx[warp][lane] = RQV(xs)[idx];
                        sy[warp][lane] = RQV(ys)[idx];
                        sz[warp][lane] = RQV(zs)[idx];
                    }
                }
                __syncwarp();
                const uint32_t m = (rg.y - b < 32u) ? (rg.y - b) : 32u;
                // bit t: staged point t is inside this lane's query
                uint32_t hits = 0;
                if (mine) {
                    for (uint32_t t = 0; t < m; ++t) {
                        bool in;
                        if constexpr (F32) {
                            const int r = f32_test<KT>(ctx, sp[warp][t]);
                            if (r < 0) {
                                in = is_inside<KT>(k, RQV(xs)[b + t], RQV(ys)[b + t], RQV(zs)[b + t]);
                                ++n_retests;
                            } else {
                                in = r > 0;
                            }
                        } else {
                            in = is_inside<KT>(k, sx[warp][t], sy[warp][t], sz[warp][t]);
                        }
                        if constexpr (ALGO == kStruct) hit(b + t, in);
                        else hits |= (uint32_t)in << t;
                    }
                    n_tests += m;
                }
                if constexpr (ALGO != kStruct) {
                    if (FILL) {  // every lane's hits in one coalesced store, lane after lane
                        uint32_t rem = __ballot_sync(0xffffffffu, hits != 0);
                        while (rem) {
                            const int j = __ffs(rem) - 1;
                            rem &= rem - 1;
                            const uint32_t hj = __shfl_sync(0xffffffffu, hits, j);
                            const unsigned long long o0 = __shfl_sync(0xffffffffu, base + cnt, j);
                            if ((hj >> lane) & 1u) {
                                const unsigned long long o = o0 + __popc(hj & lanemask_lt());
                                if (o < a.out_cap) a.out[o] = b + lane;
                                else overflow = true;
                            }
                        }
                    }
                    cnt += __popc(hits);
                }
                __syncwarp();
            }
            if (ALGO == kStruct && mine && open) {
                open = false;
                emit_range(rs, rg.y);
            }
            }
        };

        // root: continuationCriterion(0, 0)
        bool over = false, in = false;
        if (valid) {
            if constexpr (ALGO == kNeighbors) {
                over = box_overlap<KT>(k, RQV(centers), s_radii[0]);
            } else {
                const int j = box_intersect<KT>(k, RQV(centers), s_radii[0]);
                in = (j == kInside);
                over = (j == kOverlap);
            }
        }
        int sp_top = 0;
        {
            const uint32_t mo = __ballot_sync(0xffffffffu, over);
            const uint32_t mi = __ballot_sync(0xffffffffu, in);
            if (mo | mi) {
                const uint32_t fc0 = RQV(offsets)[0];
                const uint2 rg0 = RQV(ranges)[0];
                if (lane == 0) {
                    sn[0] = 0;
                    sf[0] = fc0;
                    sr[0] = rg0;
                    so[0] = mo;
                    si[0] = mi;
                    sd[0] = 0;
                }
                sp_top = 1;
            }
        }
        __syncwarp();
        while (sp_top > 0) {
            --sp_top;
            const uint32_t node = sn[sp_top];
            const uint32_t fc = sf[sp_top];
            const uint2 nrg = sr[sp_top];
            const uint32_t mo = so[sp_top];
            const uint32_t mi = si[sp_top];
            const uint32_t depth = sd[sp_top];
            __syncwarp();
            if constexpr (ALGO == kStruct) {
                if (mi & lbit) emit_range(nrg.x, nrg.y);
            } else if (mi) {
                // a fully-inside node: every lane of mi adds the node's whole range; the
                // warp writes it for one lane at a time, 32 consecutive indices per store
                const uint32_t len = nrg.y - nrg.x;
                if constexpr (CHUNK) {
                    if (len) {
                        uint32_t rem = mi;
                        while (rem) {
                            const int j = __ffs(rem) - 1;
                            rem &= rem - 1;
                            const ChunkPos p = chunk_reserve(j, len);
                            for (uint32_t t = lane; t < len; t += 32) chunk_store(p, t, nrg.x + t);
                        }
                    }
                } else {
                    if (FILL) {
                        uint32_t rem = mi;
                        while (rem) {
                            const int j = __ffs(rem) - 1;
                            rem &= rem - 1;
                            const unsigned long long o0 = __shfl_sync(0xffffffffu, base + cnt, j);
                            for (uint32_t t = lane; t < len; t += 32) {
                                const unsigned long long o = o0 + t;
                                if (o < a.out_cap) a.out[o] = nrg.x + t;
                                else overflow = true;
                            }
                        }
                    }
                    if (mi & lbit) cnt += len;
                }
            }
            if (mo == 0) continue;
            if (fc == 0) {
                scan_leaf(node, nrg, mo);
                continue;
            }
            const uint32_t cd = depth + 1;
            // lane j (< 8) keeps child j's first-child link, range and lane masks
            uint32_t my_fc = 0, my_mo = 0, my_mi = 0;
            uint2 my_rg = make_uint2(0u, 0u);
            if (lane < 8) {
                my_fc = RQV(offsets)[fc + lane];
                my_rg = RQV(ranges)[fc + lane];
            }
            // neighborsApprox (linear_octree.hpp:979-985): below its precision level a
            // child is cut before any box test, its whole range added in upper-bound mode
            const bool cut = ALGO == kStruct && approx_cut != 0 && cd >= approx_cut;
            {
                // child tests transposed: lane = (query slot lane / 8, child lane % 8), the
                // node's active queries four at a time, so a node that few queries of the
                // packet reach costs few passes; each lane tests with the query's own
                // SearchKernel and the child's centre, as the per-query walk does
                const int slot = lane >> 3;
                const double* ocp = RQV(centers) + 3ull * (fc + (lane & 7));
                const double oc[3] = {ocp[0], ocp[1], ocp[2]};
                uint32_t rem = mo;
                while (rem) {
                    int ql[4];
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        ql[s] = rem ? __ffs(rem) - 1 : -1;
                        rem &= rem - 1;
                    }
                    const int myq = slot == 0 ? ql[0] : slot == 1 ? ql[1] : slot == 2 ? ql[2] : ql[3];
                    bool o = false, n = false;
                    if (myq >= 0) {
                        const SearchKernel kq = kernel_of<KT>(s_qp[warp], myq);
                        if constexpr (ALGO == kNeighbors) {
                            o = box_overlap<KT>(kq, oc, s_radii[cd]);
                        } else if (cut) {
                            n = approx_upper;
                        } else {
                            const int jj = box_intersect<KT>(kq, oc, s_radii[cd]);
                            n = (jj == kInside);
                            o = (jj == kOverlap);
                        }
                    }
                    const uint32_t bo = __ballot_sync(0xffffffffu, o);
                    const uint32_t bi = __ballot_sync(0xffffffffu, n);
                    if (lane < 8) {  // bit 8 s + j of a ballot: query ql[s] against child j
#pragma unroll
                        for (int s = 0; s < 4; ++s) {
                            if (ql[s] >= 0) {
                                my_mo |= ((bo >> (8 * s + lane)) & 1u) << ql[s];
                                my_mi |= ((bi >> (8 * s + lane)) & 1u) << ql[s];
                            }
                        }
                    }
                }
            }
            if (lane < 8 && my_fc == 0 && my_rg.x == my_rg.y) {  // empty leaf: nothing to scan or add
                my_mo = 0;
                if (ALGO != kStruct) my_mi = 0;  // neighborsStruct still adds its empty range
            }
            const uint32_t pushm = __ballot_sync(0xffffffffu, lane < 8 && (my_mo | my_mi) != 0);
            const int np = __popc(pushm);
            if (sp_top + np > kPkStack) {
                overflow = true;
                break;
            }
            if ((pushm >> lane) & 1u) {
                // lowest octant on top of the stack
                const int slot = sp_top + __popc(pushm >> (lane + 1));
                sn[slot] = fc + lane;
                sf[slot] = my_fc;
                sr[slot] = my_rg;
                so[slot] = my_mo;
                si[slot] = my_mi;
                sd[slot] = (uint8_t)cd;
            }
            __syncwarp();
            sp_top += np;
        }
        if (overflow) set_err(a.err, (FILL && !CHUNK) ? kErrOutputCapacity : kErrStackOverflow);
        if (CHUNK && ck_over) set_err(a.err, kErrChunkCapacity);
        if ((!FILL || CHUNK) && valid) {
            a.counts[qi] = cnt;
            if (CHUNK) a.chunk_first[qi] = ck_first;
            if (ALGO == kStruct) a.counts2[qi] = cnt2;
        }
        __syncwarp();
    }
    if (a.stats) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            n_tests += __shfl_down_sync(0xffffffffu, n_tests, off);
            n_retests += __shfl_down_sync(0xffffffffu, n_retests, off);
        }
        if (lane == 0) {
            atomicAdd(&a.stats[0], n_tests);
            atomicAdd(&a.stats[1], n_retests);
        }
    }
}

// FP32 leaf-relative coordinates: one warp per node; leaves write their points.
__global__ void k_leaf_rel(const double* __restrict__ xs, const double* __restrict__ ys,
                           const double* __restrict__ zs, const uint32_t* __restrict__ offsets,
                           const uint2* __restrict__ ranges, const double* __restrict__ centers, uint32_t n_total,
                           float4* __restrict__ rel) {
    const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n_total) return;
    const uint32_t node = (uint32_t)w;
    if (offsets[node] != 0) return;
    const uint2 rg = ranges[node];
    const double cx = centers[3ull * node], cy = centers[3ull * node + 1], cz = centers[3ull * node + 2];
    for (uint32_t i = rg.x + lane; i < rg.y; i += 32) {
        float4 v;
        v.x = (float)dsub(xs[i], cx);
        v.y = (float)dsub(ys[i], cy);
        v.z = (float)dsub(zs[i], cz);
        // L1 norm, rounded up so that it bounds the exact L1 norm of the FP32 (x, y, z)
        v.w = __fadd_ru(__fadd_ru(fabsf(v.x), fabsf(v.y)), fabsf(v.z));
        rel[i] = v;
    }
}

int sm_count_p(int device) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v;
}

// mode: 0 count, 1 fill at known offsets, 2 one pass into result chunks
template <int KT, int ALGO, int MULTI>
cudaError_t launch_pk_m(const PacketArgs& a, int mode, bool fp32, int grid, cudaStream_t s) {
    if constexpr (MULTI == 2 && ALGO == kStruct) {  // batches do not search neighborsStruct
        return cudaErrorInvalidValue;
    }
    if (mode == 2) {
        if constexpr (ALGO != kStruct) {
            if (fp32) k_radius_packet<KT, ALGO, true, true, MULTI, true><<<grid, kPkThreads, 0, s>>>(a);
            else k_radius_packet<KT, ALGO, true, false, MULTI, true><<<grid, kPkThreads, 0, s>>>(a);
        }
    } else if (mode == 1) {
        if (fp32) k_radius_packet<KT, ALGO, true, true, MULTI><<<grid, kPkThreads, 0, s>>>(a);
        else k_radius_packet<KT, ALGO, true, false, MULTI><<<grid, kPkThreads, 0, s>>>(a);
    } else {
        if (fp32) k_radius_packet<KT, ALGO, false, true, MULTI><<<grid, kPkThreads, 0, s>>>(a);
        else k_radius_packet<KT, ALGO, false, false, MULTI><<<grid, kPkThreads, 0, s>>>(a);
    }
    return cudaGetLastError();
}

template <int KT, int ALGO>
cudaError_t launch_pk(const PacketArgs& a, int mode, bool fp32, int grid, cudaStream_t s) {
    if (a.grp) {
        if (a.one_cloud) return launch_pk_m<KT, ALGO, 2>(a, mode, fp32, grid, s);
        return launch_pk_m<KT, ALGO, 1>(a, mode, fp32, grid, s);
    }
    return launch_pk_m<KT, ALGO, 0>(a, mode, fp32, grid, s);
}

template <int KT>
cudaError_t launch_pk_a(const PacketArgs& a, int algo, int mode, bool fp32, int grid, cudaStream_t s) {
    switch (algo) {
        case kNeighbors: return launch_pk<KT, kNeighbors>(a, mode, fp32, grid, s);
        case kStruct: return launch_pk<KT, kStruct>(a, mode, fp32, grid, s);
        default: return launch_pk<KT, kPrune>(a, mode, fp32, grid, s);
    }
}

// Each radius query's chain of result chunks into its CSR slot.  A warp takes
// S queries at a time (S from 4 up to 32, as many as keep every warp busy):
// their counts, offsets and first chunks come in one coalesced round trip; then
// the chains of kCompactBatch queries are walked in lockstep, each step loading
// one chunk of every one of them (and their next links) before storing any, so
// the four latency chains overlap.
constexpr int kCompactBatch = 4;
static_assert(kChunk == 64, "a chunk is two 32-entry rows");

__global__ void __launch_bounds__(256) k_chunk_compact(const unsigned long long* __restrict__ counts,
                                                       const unsigned long long* __restrict__ offs,
                                                       const uint32_t* __restrict__ first,
                                                       const uint32_t* __restrict__ next,
                                                       const uint32_t* __restrict__ pool, uint64_t chunk_cap,
                                                       uint32_t* __restrict__ out, uint64_t out_cap, uint64_t n,
                                                       const uint64_t* d_n, uint32_t* err) {
    if (d_n) n = *d_n;
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    uint32_t S = kCompactBatch;
    while (S < 32 && (uint64_t)S * nwarps < n) S <<= 1;
    bool bad = false;  // a chain cut short by a pool overflow (reported by the search kernel), or no room
    for (uint64_t q0 = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * S; q0 < n; q0 += nwarps * S) {
        const uint64_t q = q0 + lane;
        unsigned long long cnt = 0, o = 0;
        uint32_t c0 = kNoChunk;
        if ((uint32_t)lane < S && q < n) {
            cnt = counts[q];
            if (cnt) {
                o = offs[q];
                c0 = first[q];
            }
        }
        uint32_t todo = __ballot_sync(0xffffffffu, cnt != 0);
        while (todo) {
            unsigned long long cj[kCompactBatch], dst[kCompactBatch], done[kCompactBatch];
            uint32_t cur[kCompactBatch];
#pragma unroll
            for (int b = 0; b < kCompactBatch; ++b) {
                const int j = todo ? __ffs(todo) - 1 : -1;
                todo &= todo - 1;
                const unsigned long long cb = __shfl_sync(0xffffffffu, cnt, j & 31);
                cj[b] = j >= 0 ? cb : 0ull;
                dst[b] = __shfl_sync(0xffffffffu, o, j & 31);
                cur[b] = __shfl_sync(0xffffffffu, c0, j & 31);
                done[b] = 0;
            }
            for (;;) {  // one chunk of every unfinished chain per step (warp-uniform)
                bool any = false;
#pragma unroll
                for (int b = 0; b < kCompactBatch; ++b) any = any || done[b] < cj[b];
                if (!any) break;
                uint32_t v[kCompactBatch][2], nx[kCompactBatch];
#pragma unroll
                for (int b = 0; b < kCompactBatch; ++b) {
                    v[b][0] = v[b][1] = 0;
                    nx[b] = kNoChunk;
                    if (done[b] < cj[b] && cur[b] < chunk_cap) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const uint32_t t = 32u * h + lane;
                            if (done[b] + t < cj[b]) v[b][h] = pool[(uint64_t)cur[b] * kChunk + t];
                        }
                        if (done[b] + kChunk < cj[b]) nx[b] = next[cur[b]];
                    }
                }
#pragma unroll
                for (int b = 0; b < kCompactBatch; ++b) {
                    if (done[b] >= cj[b]) continue;
                    if (cur[b] >= chunk_cap) {
                        bad = true;
                        done[b] = cj[b];
                        continue;
                    }
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const uint32_t t = 32u * h + lane;
                        if (done[b] + t < cj[b]) {
                            const unsigned long long w = dst[b] + done[b] + t;
                            if (w < out_cap) out[w] = v[b][h];
                            else bad = true;
                        }
                    }
                    done[b] = (cj[b] - done[b] > kChunk) ? done[b] + kChunk : cj[b];
                    cur[b] = nx[b];
                }
            }
        }
    }
    if (bad) set_err(err, kErrOutputCapacity);
}

// One warp per query: the sum of mix64 over the query's result chain (the
// count is the search's), instead of moving the chain into a CSR array.
__global__ void __launch_bounds__(256) k_chunk_hash(const unsigned long long* __restrict__ counts,
                                                    const uint32_t* __restrict__ first,
                                                    const uint32_t* __restrict__ next,
                                                    const uint32_t* __restrict__ pool, uint64_t chunk_cap,
                                                    unsigned long long* __restrict__ hashes, uint64_t n,
                                                    uint32_t* err) {
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t q = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < n; q += nwarps) {
        const unsigned long long cnt = counts[q];
        unsigned long long h = 0;
        uint32_t c = first[q];
        bool bad = false;
        for (unsigned long long done = 0; done < cnt;) {
            if (c >= chunk_cap) {  // a chain cut short by a pool overflow (reported by the search kernel)
                bad = true;
                break;
            }
            const unsigned long long m = (cnt - done < kChunk) ? (cnt - done) : kChunk;
            for (uint32_t t = lane; t < m; t += 32) h += mix64(pool[(uint64_t)c * kChunk + t]);
            done += m;
            if (done < cnt) c = next[c];
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) h += __shfl_xor_sync(0xffffffffu, h, off);
        if (lane == 0) hashes[q] = h;
        if (bad && lane == 0) set_err(err, kErrOutputCapacity);
    }
}

}  // namespace

// FP32 (x, y, z) of every point relative to the box centre, each rounded once
// from the FP64 difference; w = 0.
__global__ void k_center_rel(const double* __restrict__ xs, const double* __restrict__ ys,
                             const double* __restrict__ zs, const BoxD* __restrict__ box, uint64_t n,
                             float4* __restrict__ out) {
    const double cx = box->center[0], cy = box->center[1], cz = box->center[2];
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = make_float4((float)dsub(xs[i], cx), (float)dsub(ys[i], cy), (float)dsub(zs[i], cz), 0.0f);
}

cudaError_t launch_center_rel(Cloud& c) {
    cudaError_t e;
    if ((e = c.crel.reserve(16 * (c.n ? c.n : 1))) != cudaSuccess) return e;
    if (c.n == 0) return cudaSuccess;
    const uint64_t want = (c.n + 255) / 256;
    const unsigned grid = (unsigned)(want < 148ull * 16 ? want : 148ull * 16);
    k_center_rel<<<grid, 256, 0, c.stream>>>(c.xs.as<double>(), c.ys.as<double>(), c.zs.as<double>(),
                                             c.d_box.as<BoxD>(), c.n, c.crel.as<float4>());
    return cudaGetLastError();
}

cudaError_t launch_leaf_rel(Cloud& c) {
    cudaError_t e;
    if ((e = c.rel.reserve(16 * (c.n ? c.n : 1))) != cudaSuccess) return e;
    if (c.n == 0 || c.n_total == 0) return cudaSuccess;
    const uint64_t threads = 32ull * c.n_total;
    k_leaf_rel<<<(unsigned)((threads + 255) / 256), 256, 0, c.stream>>>(
        c.xs.as<double>(), c.ys.as<double>(), c.zs.as<double>(), c.offsets.as<uint32_t>(), c.ranges.as<uint2>(),
        c.centers.as<double>(), c.n_total, c.rel.as<float4>());
    return cudaGetLastError();
}

CloudView cloud_view(const Cloud& c) {
    CloudView v;
    v.xs = c.xs.as<double>();
    v.ys = c.ys.as<double>();
    v.zs = c.zs.as<double>();
    v.rel = c.rel.as<float4>();
    v.crel = c.crel_built ? c.crel.as<float4>() : nullptr;
    v.offsets = c.offsets.as<uint32_t>();
    v.ranges = c.ranges.as<uint2>();
    v.centers = c.centers.as<double>();
    v.geom = reinterpret_cast<const LevelGeom*>(c.d_box.as<unsigned char>() + sizeof(BoxD));
    v.box = c.d_box.as<BoxD>();
    v.encoder = c.params.encoder;
    v.pad = 0;
    return v;
}

cudaError_t launch_radius_table(int device, cudaStream_t s, int kernel, int algo, int mode, bool fp32,
                                const DynGroup* d_grp, const SearchReq* single, uint64_t packets,
                                const uint32_t* d_order, unsigned long long* d_counts, unsigned long long* d_counts2,
                                const unsigned long long* d_offsets, uint32_t* d_out, uint64_t out_capacity,
                                uint32_t* d_packet_ctr, unsigned long long* d_stats, uint32_t* d_err,
                                int blocks_per_sm, const ChunkArgs* chunks) {
    cudaError_t e;
    if (!d_grp && packets == 0) return cudaSuccess;
    if ((e = cudaMemsetAsync(d_packet_ctr, 0, 4, s)) != cudaSuccess) return e;
    PacketArgs a;
    a.single = single ? *single : SearchReq{};
    a.grp = d_grp;
    a.one_cloud = d_grp != nullptr && single != nullptr;  // a batch on one cloud: its view in `single`
    a.packets = packets;
    a.order = d_order;
    a.counts = d_counts;
    a.counts2 = d_counts2;
    a.offs = d_offsets;
    a.out = d_out;
    a.out_cap = out_capacity;
    a.packet_ctr = d_packet_ctr;
    a.stats = d_stats;
    a.err = d_err;
    a.chunk_pool = chunks ? chunks->pool : nullptr;
    a.chunk_next = chunks ? chunks->next : nullptr;
    a.chunk_first = chunks ? chunks->first : nullptr;
    a.chunk_ctr = chunks ? chunks->ctr : nullptr;
    a.chunk_cap = chunks ? chunks->cap : 0;
    if (mode == 2 && (!chunks || algo == kStruct)) return cudaErrorInvalidValue;
    // persistent grid: warps take packets from the counter until none is left
    const uint64_t cap = (uint64_t)sm_count_p(device) * (blocks_per_sm > 0 ? blocks_per_sm : 12);
    const uint64_t want = d_grp ? cap : (packets + kPkWarps - 1) / kPkWarps;
    const int grid = (int)(want < cap ? want : cap);
    switch (kernel) {
        case kCircle: return launch_pk_a<kCircle>(a, algo, mode, fp32, grid, s);
        case kSquare: return launch_pk_a<kSquare>(a, algo, mode, fp32, grid, s);
        case kCube: return launch_pk_a<kCube>(a, algo, mode, fp32, grid, s);
        default: return launch_pk_a<kSphere>(a, algo, mode, fp32, grid, s);
    }
}

cudaError_t launch_chunk_hash(int device, cudaStream_t s, const unsigned long long* d_counts, const ChunkArgs& chunks,
                              unsigned long long* d_hashes, uint64_t n, uint32_t* d_err) {
    if (n == 0) return cudaSuccess;
    const uint64_t cap = (uint64_t)sm_count_p(device) * 8;
    const uint64_t want = (n + 7) / 8;
    const int grid = (int)(want < cap ? want : cap);
    k_chunk_hash<<<grid, 256, 0, s>>>(d_counts, chunks.first, chunks.next, chunks.pool, chunks.cap, d_hashes, n,
                                      d_err);
    return cudaGetLastError();
}

cudaError_t launch_chunk_compact(int device, cudaStream_t s, const unsigned long long* d_counts,
                                 const unsigned long long* d_offsets, const ChunkArgs& chunks, uint32_t* d_out,
                                 uint64_t out_capacity, uint64_t n, const uint64_t* d_n, uint32_t* d_err) {
    if (!d_n && n == 0) return cudaSuccess;
    const uint64_t cap = (uint64_t)sm_count_p(device) * 8;
    const uint64_t want = d_n ? cap : (n + 31) / 32;  // 8 warps of at least 4 queries per block
    const int grid = (int)(want < cap ? (want ? want : 1) : cap);
    k_chunk_compact<<<grid, 256, 0, s>>>(d_counts, d_offsets, chunks.first, chunks.next, chunks.pool, chunks.cap,
                                         d_out, out_capacity, n, d_n, d_err);
    return cudaGetLastError();
}

cudaError_t launch_radius_packet(Cloud& c, int kernel, int algo, int mode, bool fp32, const double* d_centers,
                                 uint64_t nq, const double* d_radii, double radius, const uint32_t* d_order,
                                 unsigned long long* d_counts, unsigned long long* d_counts2,
                                 const unsigned long long* d_offsets, uint32_t* d_out, uint64_t out_capacity,
                                 const ChunkArgs* chunks) {
    cudaError_t e;
    if (nq == 0) return cudaSuccess;
    if ((e = c.packet_ctr.reserve(256)) != cudaSuccess) return e;
    SearchReq r{};
    r.cv = cloud_view(c);
    r.centers = d_centers;
    r.radii = d_radii;
    r.radius = radius;
    r.q_begin = 0;
    r.q_end = nq;
    r.packet_begin = 0;
    r.out_begin = 0;
    r.k = 0;
    r.cloud_id = 0;
    r.approx_cut = c.approx_cut;
    r.approx_upper = (uint32_t)c.approx_upper;
    KernelClock clk(c, 0);
    e = launch_radius_table(c.device, c.stream, kernel, algo, mode, fp32, nullptr, &r, (nq + 31) / 32, d_order,
                            d_counts, d_counts2, d_offsets, d_out, out_capacity, c.packet_ctr.as<uint32_t>(),
                            c.stats.as<unsigned long long>(), c.d_err.as<uint32_t>(), 0, chunks);
    clk.stop();
    return e;
}

// A kernel of this file's device code, for preload_kernels.
const void* kernel_anchor_radius_packet() { return reinterpret_cast<const void*>(&k_center_rel); }

}  // namespace octb
