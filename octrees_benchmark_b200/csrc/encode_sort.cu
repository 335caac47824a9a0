// Bounding box, SFC encoding and the stable key sort with point reorder.
//
// Reference path replaced: PointEncoder::sortPoints (inc/encoding/point_encoder.hpp:
// 285-383, 484-503): mbb (inc/geometry/box.hpp:95-137) -> encodePoints -> an
// 8 x 8-bit LSD radix sort that moves keys and points together.
//
// B200 design:
//  * k_bbox: one pass over the AoS input, block min/max, the last block folds
//    the partials and writes the Box and the per-level geometry.
//  * k_encode: anchor coordinates + Morton/Hilbert key per point (Hilbert: the
//    24-state automaton walked two levels per shared-memory lookup), and in the
//    same pass the 8 digit histograms of every key (so no pass re-reads keys
//    to count).
//  * k_onesweep: one kernel per 8-bit digit, single-pass "onesweep" radix
//    scatter: each 3072-key tile ranks its keys stably in shared memory (the
//    lanes holding the same digit found by 8 ballots, per-warp counters),
//    publishes its digit counts, resolves its
//    global digit offsets by decoupled look-back over the preceding tiles
//    (bounded waits), and writes keys and 32-bit point ids out digit-grouped,
//    which keeps the writes coalesced.  Digits equal for every key are
//    skipped.  Values are generated on the fly in the first pass.
//  * k_gather: reorders the coordinates into SoA float64 arrays.
#include <cfloat>
#include <cstddef>
#include <mutex>

#include "cloud.h"
#include "sfc.cuh"

namespace octb {

namespace {

constexpr int kBboxThreads = 256;
constexpr int kEncThreads = 256;
// onesweep tiles: 8 keys per thread x 384 threads, 3 blocks per SM (measured on 10M keys, 8
// passes: 112 us per pass against 128 us for 16 x 256, 4096-key tiles)
constexpr int kSortThreads = 384;
constexpr int kSortItems = 12;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4608 keys
constexpr int kSortWarps = kSortThreads / 32;
// resident onesweep blocks per SM (registers: 12 keys and values per thread; 3 blocks of
// 384 x 8 keys measured 1.8 % slower on the 10M-point build)
constexpr int kSortBlocksPerSM = 2;
static_assert(kSortThreads >= 256, "threads 0..255 own one digit each");
// predecessor tiles a digit's look-back reads per round trip
constexpr int kLookAhead = 4;
constexpr int kEncGridPerSM = 4;

// look-back status word: flag (2 bits) | epoch (22 bits) | count (40 bits)
constexpr unsigned long long kFlagLocal = 1ull << 62;
constexpr unsigned long long kFlagPrefix = 2ull << 62;
constexpr unsigned long long kCountMask = (1ull << 40) - 1;
constexpr int kEpochShift = 40;
constexpr unsigned long long kEpochMask = ((1ull << 22) - 1) << kEpochShift;

struct BoxGeom {
    BoxD box;
    LevelGeom geom;
};

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_volatile_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__global__ void __launch_bounds__(kBboxThreads) k_bbox(const double* __restrict__ xyz, uint64_t n,
                                                       double* __restrict__ partial, uint32_t* ctr,
                                                       BoxGeom* out) {
    double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
    double mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // two points per thread and step: three aligned 16-byte loads (x0 y0 | z0 x1 | y1 z1);
    // a buffer that is not 16-byte aligned takes the scalar loop
    const bool vec = (reinterpret_cast<uintptr_t>(xyz) & 15u) == 0;
    const uint64_t npairs = vec ? n / 2 : 0;
    const double2* xyz2 = reinterpret_cast<const double2*>(xyz);
    for (uint64_t i = vec ? n : (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[a] = smin(mn[a], xyz[3 * i + a]);
            mx[a] = smax(mx[a], xyz[3 * i + a]);
        }
    }
    // four pairs per thread and step (12 independent 16-byte loads in flight)
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < npairs; t += 4 * stride) {
        double2 v[4][3];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint64_t tu = t + (uint64_t)u * stride;
            if (tu < npairs) {
                v[u][0] = xyz2[3 * tu];
                v[u][1] = xyz2[3 * tu + 1];
                v[u][2] = xyz2[3 * tu + 2];
            } else {  // repeat a pair already read: min / max unchanged
                v[u][0] = v[0][0];
                v[u][1] = v[0][1];
                v[u][2] = v[0][2];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double e6[6] = {v[u][0].x, v[u][0].y, v[u][1].x, v[u][1].y, v[u][2].x, v[u][2].y};
#pragma unroll
            for (int e = 0; e < 6; ++e) {
                mn[e % 3] = smin(mn[e % 3], e6[e]);  // std::min(localMin, p)
                mx[e % 3] = smax(mx[e % 3], e6[e]);  // std::max(localMax, p)
            }
        }
    }
    if (vec && (n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[a] = smin(mn[a], xyz[3 * (n - 1) + a]);
            mx[a] = smax(mx[a], xyz[3 * (n - 1) + a]);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[a] = smin(mn[a], __shfl_down_sync(0xffffffffu, mn[a], off));
            mx[a] = smax(mx[a], __shfl_down_sync(0xffffffffu, mx[a], off));
        }
    }
    __shared__ double s[kBboxThreads / 32][6];
    __shared__ bool last;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) { s[warp][a] = mn[a]; s[warp][3 + a] = mx[a]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBboxThreads / 32; ++w)
            for (int a = 0; a < 3; ++a) {
                s[0][a] = smin(s[0][a], s[w][a]);
                s[0][3 + a] = smax(s[0][3 + a], s[w][3 + a]);
            }
        for (int a = 0; a < 6; ++a) partial[6 * blockIdx.x + a] = s[0][a];
        __threadfence();
        last = (atomicAdd(ctr, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last block folds the blocks' partials with all its threads (one thread alone
    // waited for the grid's ~450 partials one L2 round trip at a time)
    double gmn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, gmx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            gmn[a] = smin(gmn[a], __ldcg(&partial[6 * b + a]));
            gmx[a] = smax(gmx[a], __ldcg(&partial[6 * b + 3 + a]));
        }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            gmn[a] = smin(gmn[a], __shfl_down_sync(0xffffffffu, gmn[a], off));
            gmx[a] = smax(gmx[a], __shfl_down_sync(0xffffffffu, gmx[a], off));
        }
    }
    if (lane == 0)
        for (int a = 0; a < 3; ++a) { s[warp][a] = gmn[a]; s[warp][3 + a] = gmx[a]; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int w = 0; w < kBboxThreads / 32; ++w)
        for (int a = 0; a < 3; ++a) {
            gmn[a] = smin(gmn[a], s[w][a]);
            gmx[a] = smax(gmx[a], s[w][3 + a]);
        }
    // Box(pair{min, max}) then Box(center, radii) (box.hpp:17-21, point_encoder.hpp:492-494)
    BoxGeom bg;
    for (int a = 0; a < 3; ++a) {
        const double r = ddiv(dsub(gmx[a], gmn[a]), 2.0);
        const double c = dadd(gmn[a], ddiv(dsub(gmx[a], gmn[a]), 2.0));
        bg.box.center[a] = c;
        bg.box.radii[a] = r;
        bg.box.min[a] = dsub(c, r);
        bg.box.max[a] = dadd(c, r);
    }
    // LinearOctree::setupBbox (linear_octree.hpp:439-455): half = 0.5f * eps * (max - min)
    const double eps = 4.76837158203125e-07;  // (double)(1.0f / 2^21)
    for (int a = 0; a < 3; ++a) bg.geom.half[a] = dmul(dmul(0.5, eps), dsub(bg.box.max[a], bg.box.min[a]));
    for (uint32_t l = 0; l <= kMaxDepth; ++l)
        for (int a = 0; a < 3; ++a) bg.geom.radii[l][a] = dmul((double)(1u << (kMaxDepth - l)), bg.geom.half[a]);
    *out = bg;
    *ctr = 0;
}

// LOW: the histograms of all 8 digits; otherwise of the upper 4 only (the split
// sort, which sorts the lower halves only inside runs, and counts its long
// runs' digits itself).
template <int ENC, bool LOW = true>
__global__ void __launch_bounds__(kEncThreads) k_encode(const double* __restrict__ xyz, uint64_t n,
                                                        const BoxGeom* __restrict__ bg, uint64_t* __restrict__ keys,
                                                        SortCtl* ctl) {
    __shared__ uint32_t hist[8 * 256];
    __shared__ uint8_t htbl[kHilbertStates * 8];
    __shared__ uint16_t htbl2[ENC == 5 ? kHilbertTable2Size : 1];
    for (int j = threadIdx.x; j < 8 * 256; j += blockDim.x) hist[j] = 0;
    if constexpr (ENC == 5) {
        for (int j = threadIdx.x; j < kHilbertStates * 8; j += blockDim.x) htbl[j] = kHilbertTable[j];
        hilbert_table2_fill(htbl2, threadIdx.x, blockDim.x);
    }
    const double c0 = bg->box.center[0], c1 = bg->box.center[1], c2 = bg->box.center[2];
    const double r0 = bg->box.radii[0], r1 = bg->box.radii[1], r2 = bg->box.radii[2];
    const double i0 = __drcp_rn(dmul(2.0, r0)), i1 = __drcp_rn(dmul(2.0, r1)), i2 = __drcp_rn(dmul(2.0, r2));
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    auto key_of = [&](double px, double py, double pz) {
        const uint32_t ax = anchor_coord_fast(px, c0, r0, i0);
        const uint32_t ay = anchor_coord_fast(py, c1, r1, i1);
        const uint32_t az = anchor_coord_fast(pz, c2, r2, i2);
        const uint64_t k = (ENC == 5) ? hilbert_encode_tbl2(ax, ay, az, htbl, htbl2) : morton_encode(ax, ay, az);
#pragma unroll
        for (int p = LOW ? 0 : 4; p < 8; ++p) atomicAdd(&hist[p * 256 + (uint32_t)((k >> (8 * p)) & 255u)], 1u);
        return k;
    };
    // two points per thread and step: three aligned 16-byte loads, one 16-byte store;
    // buffers that are not 16-byte aligned take the scalar loop
    const bool vec = ((reinterpret_cast<uintptr_t>(xyz) | reinterpret_cast<uintptr_t>(keys)) & 15u) == 0;
    const uint64_t npairs = vec ? n / 2 : 0;
    for (uint64_t i = vec ? n : (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = key_of(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        keys[i] = k;
    }
    const double2* xyz2 = reinterpret_cast<const double2*>(xyz);
    ulonglong2* keys2 = reinterpret_cast<ulonglong2*>(keys);
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < npairs; t += stride) {
        const double2 a = xyz2[3 * t], b = xyz2[3 * t + 1], c = xyz2[3 * t + 2];
        ulonglong2 kk;
        kk.x = key_of(a.x, a.y, b.x);
        kk.y = key_of(b.y, c.x, c.y);
        keys2[t] = kk;
    }
    if (vec && (n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const uint64_t k = key_of(xyz[3 * (n - 1)], xyz[3 * (n - 1) + 1], xyz[3 * (n - 1) + 2]);
        keys[n - 1] = k;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < 8 * 256; j += blockDim.x) {
        const uint32_t v = hist[j];
        if (v) atomicAdd(&ctl->hist[j >> 8][j & 255], v);
    }
}

// Exclusive scans of the 8 histograms; pass p is skipped when one digit holds
// every key.  One block of 256 threads.
__global__ void __launch_bounds__(256) k_scan_hist(SortCtl* ctl, uint64_t n, const uint64_t* d_n = nullptr) {
    __shared__ unsigned long long warp_sum[8];
    if (d_n) n = *d_n;
    const int d = threadIdx.x, lane = d & 31, warp = d >> 5;
    for (int p = 0; p < 8; ++p) {
        const unsigned long long v = ctl->hist[p][d];
        unsigned long long x = v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        if (lane == 31) warp_sum[warp] = x;
        const bool full = (v == n);
        const int any_full = __syncthreads_or(full);
        unsigned long long base = 0;
        for (int w = 0; w < warp; ++w) base += warp_sum[w];
        ctl->offs[p][d] = base + x - v;
        if (d == 0) {
            ctl->skip[p] = any_full ? 1u : 0u;
            ctl->tile_ctr[p] = 0;
        }
        __syncthreads();
    }
}

// K: uint64_t (the full keys; digit `pass` is bits 8 pass .. 8 pass + 7) or
// uint32_t (the upper key halves; digit `pass` (4..7) is bits 8 pass - 32 ..).
// V: uint32_t (the input position) or uint64_t (the lower key half << 32 | the
// input position; the first pass reads both halves from `lo_src`, the whole
// keys in input order, and no `kin`).
template <bool FIRST, class K = uint64_t, class V = uint32_t>
__global__ void __launch_bounds__(kSortThreads, kSortBlocksPerSM) k_onesweep(const K* __restrict__ kin,
                                                           const V* __restrict__ vin,
                                                           K* __restrict__ kout, V* __restrict__ vout,
                                                           uint64_t n, int pass, SortCtl* ctl,
                                                           unsigned long long* status, uint32_t epoch,
                                                           uint32_t* err, const uint64_t* d_n = nullptr,
                                                           const uint32_t* d_epoch = nullptr,
                                                           const uint64_t* __restrict__ lo_src = nullptr) {
    extern __shared__ __align__(16) unsigned char smem[];
    V* svals = reinterpret_cast<V*>(smem);                                     // kSortTile
    K* skeys = reinterpret_cast<K*>(svals + kSortTile);                        // kSortTile
    uint32_t* wcnt = reinterpret_cast<uint32_t*>(skeys + kSortTile);           // kSortWarps x 256
    uint32_t* tstart = wcnt + kSortWarps * 256;                                // 256
    unsigned long long* gbase = reinterpret_cast<unsigned long long*>(tstart + 256);  // 256
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_wsum[kSortWarps];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int shift = 8 * pass - (sizeof(K) == 4 ? 32 : 0);
    // sizes set on the device (batched launches): key count, and the epoch base
    // of this batch's passes
    if (d_n) n = *d_n;
    if (d_epoch) epoch = (*d_epoch + (uint32_t)pass) & ((1u << 22) - 1);
    const uint64_t ntiles = (n + kSortTile - 1) / kSortTile;
    // persistent: a block takes tiles in order until none is left; a tile only
    // waits on lower tiles, which running blocks hold
    for (;;) {
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_ctr[pass], 1u);
    for (int j = tid; j < kSortWarps * 256; j += kSortThreads) wcnt[j] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    if ((uint64_t)tile >= ntiles) break;
    const uint64_t base = (uint64_t)tile * kSortTile;

    K k[kSortItems];
    V v[kSortItems];
    uint32_t rank[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const uint64_t idx = base + (uint64_t)warp * (32 * kSortItems) + (uint64_t)j * 32 + lane;
        const bool valid = idx < n;
        if constexpr (FIRST && sizeof(V) == 8) {  // the split sort's first pass reads the whole keys only
            const uint64_t whole = valid ? lo_src[idx] : ~0ull;
            k[j] = (K)(whole >> 32);
            v[j] = (whole << 32) | (uint64_t)(uint32_t)idx;
        } else {
            k[j] = valid ? kin[idx] : (K)~0ull;
        }
        if (FIRST) {
            if constexpr (sizeof(V) != 8) v[j] = (V)(uint32_t)idx;
        } else {
            v[j] = valid ? vin[idx] : (V)0;
        }
    }
    // stable rank inside the warp: item j of lane l precedes item j of lane l+1,
    // and every item j precedes item j+1.  The lanes holding the same digit are
    // found with 8 ballots (one per digit bit); the highest of them updates the
    // warp's counter for all.
    uint32_t* cnt = wcnt + warp * 256;
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const uint64_t idx = base + (uint64_t)warp * (32 * kSortItems) + (uint64_t)j * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = (uint32_t)((k[j] >> shift) & 255u);
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const uint32_t bal = __ballot_sync(0xffffffffu, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? bal : ~bal;
        }
        const int leader = 31 - __clz(peers);  // -1 only for an invalid lane with no valid peer
        uint32_t before = 0;
        if (valid && lane == leader) {
            before = cnt[d];
            cnt[d] = before + __popc(peers);
        }
        __syncwarp();
        before = __shfl_sync(0xffffffffu, before, leader & 31);
        rank[j] = before + __popc(peers & lanemask_lt());
    }
    __syncthreads();
    // per digit (threads 0..255): warp prefixes and the tile total
    const int d = tid;
    uint32_t total = 0;
    if (d < 256) {
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = wcnt[w * 256 + d];
            wcnt[w * 256 + d] = total;
            total += c;
        }
    }
    const unsigned long long ep = ((unsigned long long)epoch << kEpochShift) & kEpochMask;
    unsigned long long* my = status + (uint64_t)tile * 256 + (d & 255);
    if (d < 256) st_volatile_u64(my, (tile == 0 ? kFlagPrefix : kFlagLocal) | ep | (unsigned long long)total);
    // tile-local exclusive scan of totals over digits (digits live in warps 0..7)
    {
        uint32_t x = total;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        if (lane == 31 && warp < 8) s_wsum[warp] = x;
        __syncthreads();
        uint32_t pre = 0;
        if (d < 256) {
            for (int w = 0; w < warp; ++w) pre += s_wsum[w];
            tstart[d] = pre + x - total;
        }
    }
    // decoupled look-back over the preceding tiles (bounded wait); each round
    // reads kLookAhead predecessors at once and sums them nearest first up to
    // the first prefix, or up to one that has not published
    unsigned long long excl = 0;
    if (d < 256 && tile > 0) {
        int64_t t = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (t >= 0) {
            unsigned long long s[kLookAhead];
#pragma unroll
            for (int q = 0; q < kLookAhead; ++q)  // tile 0 is a prefix: a walk never passes below it
                s[q] = (t - q >= 0) ? ld_volatile_u64(status + (uint64_t)(t - q) * 256 + d) : 0ull;
            int used = 0;
            bool found = false;
#pragma unroll
            for (int q = 0; q < kLookAhead; ++q) {
                const unsigned long long flag = s[q] & (3ull << 62);
                if ((s[q] & kEpochMask) != ep || flag == 0) break;
                excl += s[q] & kCountMask;
                ++used;
                if (flag == kFlagPrefix) {
                    found = true;
                    break;
                }
            }
            if (found) break;
            t -= used;
            if (used == 0) {
                if (++spins > kSpinLimit) {
                    set_err(err, kErrSpinLimit);
                    break;
                }
                __nanosleep(32);
            }
        }
        st_volatile_u64(my, kFlagPrefix | ep | (excl + total));
    }
    if (d < 256) gbase[d] = ctl->offs[pass][d] + excl;
    __syncthreads();
    // scatter into shared memory in digit order
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const uint64_t idx = base + (uint64_t)warp * (32 * kSortItems) + (uint64_t)j * 32 + lane;
        if (idx < n) {
            const uint32_t dd = (uint32_t)((k[j] >> shift) & 255u);
            const uint32_t pos = tstart[dd] + wcnt[warp * 256 + dd] + rank[j];
            skeys[pos] = k[j];
            svals[pos] = v[j];
        }
    }
    __syncthreads();
    const uint32_t cnt_tile = (uint32_t)((n - base) < (uint64_t)kSortTile ? (n - base) : (uint64_t)kSortTile);
    for (uint32_t s = tid; s < cnt_tile; s += kSortThreads) {
        const K key = skeys[s];
        const uint32_t dd = (uint32_t)((key >> shift) & 255u);
        const unsigned long long o = gbase[dd] + (s - tstart[dd]);
        if (o < n) {  // always true unless a look-back gave up (then err is set)
            kout[o] = key;
            vout[o] = svals[s];
        }
    }
    __syncthreads();  // shared memory and s_tile are reused by the next tile
    }
}

// ---------------------------------------------------------------------------
// Sort on the upper key halves, then the runs of equal upper halves by the
// lower halves.  A stable order by the upper 32 bits (4 onesweep passes on
// 32-bit keys: 16 bytes per key and pass instead of 24) leaves the points of
// each run (equal upper halves: one cell at depth ~10.7) in input order; a
// stable order of each run by its full keys then gives the stable order of the
// whole 63-bit keys, which is the reference's (point_encoder.hpp:285-383).
// Runs are mostly short (a 10M-point 1.5 km tile: a few points), so a thread
// places each point of a run of up to kRunSmall points, a warp or a block sorts
// a run of up to kRunMid in shared memory (bitonic over (low half, position in
// run): unique, so the order is stable), and the runs longer than that (dense
// clusters) are compacted and sorted by (run, lower half) with onesweep passes
// of their own (launch_sort_long).  The same kernels write the sorted keys, the
// permutation and the reordered SoA coordinates.
// ---------------------------------------------------------------------------
constexpr uint32_t kRunSmall = 32;
constexpr uint32_t kRunWarp = 256;   // runs a warp sorts (kRunSmall < len <= kRunWarp)
constexpr uint32_t kRunMid = 4096;   // runs a block sorts (kRunWarp < len <= kRunMid)
constexpr int kRunMidThreads = 512;  // 4 blocks (32 KB of shared memory each) per SM
constexpr int kRunWarpThreads = 256;

// Runs for k_runs_warp are listed from the front of the run list, runs for
// k_runs_mid from its back (both as (start, length) pairs).
struct RunCtl {
    uint32_t w_count, w_next;  // warp runs listed, and k_runs_warp's work counter
    uint32_t b_count, b_next;  // block runs listed, and k_runs_mid's work counter
    uint32_t big;              // a run longer than kRunMid was found
    uint32_t cap;              // entries of the run list
    // runs longer than kRunMid listed (high 32 bits) and their points (low 32 bits), taken
    // together by one atomic, so a run's slot and its place among the compacted points
    // follow the same order (slot r's points come after those of every slot below r)
    unsigned long long l_packed;
};
static_assert(sizeof(RunCtl) == 32 && offsetof(RunCtl, l_packed) == 24, "the host reads RunCtl as 8 u32");

// A run longer than kRunMid: its first point, length, and where its points sit
// in the compacted arrays of all such runs (also where they sit once those are
// sorted by (slot, lower half): the slots follow the same order).
struct LongRun {
    uint32_t start, len, off, pad;
};

// The sorted point at output position o: its key (upper half `h`, lower half
// and input position packed in `pv`), its id and its SoA coordinates.
__device__ __forceinline__ void put_sorted(uint64_t o, uint32_t h, uint64_t pv, const double* __restrict__ xyz,
                                           uint64_t* __restrict__ keys_out, uint32_t* __restrict__ perm_out,
                                           double* __restrict__ xs, double* __restrict__ ys,
                                           double* __restrict__ zs) {
    const uint32_t p = (uint32_t)pv;
    keys_out[o] = ((uint64_t)h << 32) | (pv >> 32);
    perm_out[o] = p;
    xs[o] = xyz[3ull * p];
    ys[o] = xyz[3ull * p + 1];
    zs[o] = xyz[3ull * p + 2];
}

// One thread per point.  A point of a run of at most kRunSmall points finds
// its place in the run by counting the run's points that precede it in the
// stable order (a smaller lower key half, or an equal one earlier in the run)
// and writes itself there; the first point of a longer run lists it for
// k_runs_warp / k_runs_mid (start, length), or, when it is longer than kRunMid,
// lists it for the long-run stage (k_long_*).  hi: the sorted upper halves;
// pv: lower half << 32 | input position.
// A thread takes kRunsPer points (a grid stride apart) at a time: their places
// first, then the coordinate gathers of all of them (random reads from the
// input, the kernel's DRAM traffic), then the writes, so that each thread has
// kRunsPer gathers in flight instead of one.
constexpr int kRunsPer = 4;
__global__ void __launch_bounds__(256) k_runs_small(const uint32_t* __restrict__ hi,
                                                    const uint64_t* __restrict__ pv,
                                                    const double* __restrict__ xyz, uint64_t n,
                                                    uint64_t* __restrict__ keys_out, uint32_t* __restrict__ perm_out,
                                                    double* __restrict__ xs, double* __restrict__ ys,
                                                    double* __restrict__ zs, RunCtl* rc, uint32_t* mid_list,
                                                    LongRun* __restrict__ long_list) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += kRunsPer * stride) {
        uint64_t dst[kRunsPer], val[kRunsPer];
        uint32_t hv[kRunsPer];
        bool put[kRunsPer];
#pragma unroll
        for (int u = 0; u < kRunsPer; ++u) {
            const uint64_t i = i0 + (uint64_t)u * stride;
            put[u] = false;
            dst[u] = 0;
            val[u] = 0;
            hv[u] = 0;
            if (i >= n) continue;
            const uint32_t h = hi[i];
            uint64_t s = i, e = i + 1;
            if (i > 0 && hi[i - 1] == h) {
                // inside a run: a run of more than kRunSmall points is its first point's business, and
                // two probes kRunSmall away tell (a point deep in a long run reads 3 words, not 2 x 33)
                if (i >= kRunSmall && hi[i - kRunSmall] == h) continue;
                if (i + kRunSmall < n && hi[i + kRunSmall] == h) continue;
                --s;
                while (s > 0 && hi[s - 1] == h) --s;  // the run lies within (i - kRunSmall, i + kRunSmall)
                while (e < n && hi[e] == h) ++e;
                if (e - s > kRunSmall) continue;
            } else if (i + kRunSmall < n && hi[i + kRunSmall] == h) {
                // the first point of a run of more than kRunSmall points: its end by doubling steps,
                // then bisection (hi is sorted), and the run listed by its length
                uint64_t a = i + kRunSmall + 1, b = a, step = 1;
                while (b < n && hi[b] == h) {
                    a = b + 1;
                    b += step;
                    step <<= 1;
                }
                if (b > n) b = n;
                while (a < b) {
                    const uint64_t mid = a + ((b - a) >> 1);
                    if (hi[mid] == h) a = mid + 1;
                    else b = mid;
                }
                e = a;
                if (e - s > kRunMid) {
                    const unsigned long long old = atomicAdd(&rc->l_packed, (1ull << 32) | (e - s));
                    long_list[old >> 32] = LongRun{(uint32_t)s, (uint32_t)(e - s), (uint32_t)old, 0u};
                    atomicOr(&rc->big, 1u);
                } else if (e - s <= kRunWarp) {
                    const uint32_t slot = atomicAdd(&rc->w_count, 1u);
                    mid_list[2 * slot] = (uint32_t)s;
                    mid_list[2 * slot + 1] = (uint32_t)(e - s);
                } else {
                    const uint32_t slot = rc->cap - 1u - atomicAdd(&rc->b_count, 1u);
                    mid_list[2 * slot] = (uint32_t)s;
                    mid_list[2 * slot + 1] = (uint32_t)(e - s);
                }
                continue;
            } else {
                while (e < n && hi[e] == h) ++e;  // at most kRunSmall points
            }
            const uint64_t mine = pv[i];
            const uint32_t lo = (uint32_t)(mine >> 32);
            uint64_t rank = 0;
            for (uint64_t j = s; j < e; ++j) {
                if (j == i) continue;
                const uint32_t lj = (uint32_t)(pv[j] >> 32);
                rank += (lj < lo || (lj == lo && j < i)) ? 1u : 0u;
            }
            put[u] = true;
            dst[u] = s + rank;
            val[u] = mine;
            hv[u] = h;
        }
        double px[kRunsPer], py[kRunsPer], pz[kRunsPer];
#pragma unroll
        for (int u = 0; u < kRunsPer; ++u) {
            const uint64_t p = (uint32_t)val[u];
            px[u] = put[u] ? xyz[3 * p] : 0.0;
            py[u] = put[u] ? xyz[3 * p + 1] : 0.0;
            pz[u] = put[u] ? xyz[3 * p + 2] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kRunsPer; ++u) {
            if (!put[u]) continue;
            const uint64_t o = dst[u];
            keys_out[o] = ((uint64_t)hv[u] << 32) | (val[u] >> 32);
            perm_out[o] = (uint32_t)val[u];
            xs[o] = px[u];
            ys[o] = py[u];
            zs[o] = pz[u];
        }
    }
}

// One block per listed run of kRunWarp < length <= kRunMid (persistent blocks
// take runs from a counter): bitonic sort of (lower key half << 32 | position in
// run) in shared memory - unique values, so the order is stable.
__global__ void __launch_bounds__(kRunMidThreads) k_runs_mid(const uint32_t* __restrict__ hi,
                                                             const uint64_t* __restrict__ pv,
                                                             const double* __restrict__ xyz,
                                                             uint64_t* __restrict__ keys_out,
                                                             uint32_t* __restrict__ perm_out, double* __restrict__ xs,
                                                             double* __restrict__ ys, double* __restrict__ zs,
                                                             RunCtl* rc, const uint32_t* __restrict__ mid_list) {
    __shared__ unsigned long long s[kRunMid];
    __shared__ uint32_t s_r;
    const int tid = threadIdx.x;
    const uint32_t count = rc->b_count;
    for (;;) {
        if (tid == 0) s_r = atomicAdd(&rc->b_next, 1u);
        __syncthreads();
        const uint32_t r = s_r;
        if (r >= count) break;
        const uint32_t slot = rc->cap - 1u - r;
        const uint32_t start = mid_list[2 * slot], len = mid_list[2 * slot + 1];
        uint32_t P = 64;
        while (P < len) P <<= 1;
        for (uint32_t t = tid; t < P; t += kRunMidThreads)
            s[t] = t < len ? ((pv[start + t] >> 32) << 32) | t : ~0ull;
        __syncthreads();
        for (uint32_t k = 2; k <= P; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = tid; i < P / 2; i += kRunMidThreads) {  // pair i: t and t + j
                    const uint32_t t = ((i & ~(j - 1)) << 1) | (i & (j - 1)), o = t + j;
                    const unsigned long long a = s[t], b = s[o];
                    if ((a > b) == ((t & k) == 0)) {
                        s[t] = b;
                        s[o] = a;
                    }
                }
                __syncthreads();
            }
        }
        const uint32_t h = hi[start];
        for (uint32_t t = tid; t < len; t += kRunMidThreads) {
            const uint32_t local = (uint32_t)(s[t] & 0xffffffffull);
            put_sorted(start + t, h, pv[start + local], xyz, keys_out, perm_out, xs, ys, zs);
        }
        __syncthreads();  // s and s_r are reused by the next run
    }
}

// One warp per listed run of kRunSmall < length <= kRunWarp: the same bitonic
// sort as k_runs_mid in a warp's slice of shared memory.
__global__ void __launch_bounds__(kRunWarpThreads) k_runs_warp(const uint32_t* __restrict__ hi,
                                                               const uint64_t* __restrict__ pv,
                                                               const double* __restrict__ xyz,
                                                               uint64_t* __restrict__ keys_out,
                                                               uint32_t* __restrict__ perm_out,
                                                               double* __restrict__ xs, double* __restrict__ ys,
                                                               double* __restrict__ zs, RunCtl* rc,
                                                               const uint32_t* __restrict__ mid_list) {
    __shared__ unsigned long long sw[kRunWarpThreads / 32][kRunWarp];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long* s = sw[warp];
    const uint32_t count = rc->w_count;
    for (;;) {
        uint32_t r = 0;
        if (lane == 0) r = atomicAdd(&rc->w_next, 1u);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= count) break;
        const uint32_t start = mid_list[2 * r], len = mid_list[2 * r + 1];
        uint32_t P = 64;
        while (P < len) P <<= 1;
        for (uint32_t t = lane; t < P; t += 32) s[t] = t < len ? ((pv[start + t] >> 32) << 32) | t : ~0ull;
        __syncwarp();
        for (uint32_t k = 2; k <= P; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = lane; i < P / 2; i += 32) {  // pair i: its lower element t, and t + j
                    const uint32_t t = ((i & ~(j - 1)) << 1) | (i & (j - 1)), o = t + j;
                    const unsigned long long a = s[t], b = s[o];
                    if ((a > b) == ((t & k) == 0)) {
                        s[t] = b;
                        s[o] = a;
                    }
                }
                __syncwarp();
            }
        }
        const uint32_t h = hi[start];
        for (uint32_t t = lane; t < len; t += 32) {
            const uint32_t local = (uint32_t)(s[t] & 0xffffffffull);
            put_sorted(start + t, h, pv[start + local], xyz, keys_out, perm_out, xs, ys, zs);
        }
        __syncwarp();
    }
}

// Long runs (more than kRunMid points with equal upper halves, e.g. a dense
// cluster inside one cell): their points are compacted into one array keyed by
// (run slot << 32 | lower half), sorted by the onesweep passes (stable: equal
// keys keep the run's input order), and put in place.  One block per run.
__global__ void __launch_bounds__(256) k_long_compact(const uint64_t* __restrict__ pv,
                                                      const LongRun* __restrict__ runs, const RunCtl* rc,
                                                      uint64_t* __restrict__ ckeys) {
    const uint32_t count = (uint32_t)(rc->l_packed >> 32);
    for (uint32_t r = blockIdx.x; r < count; r += gridDim.x) {
        const LongRun lr = runs[r];
        for (uint32_t t = threadIdx.x; t < lr.len; t += blockDim.x)
            ckeys[lr.off + t] = ((uint64_t)r << 32) | (pv[lr.start + t] >> 32);
    }
}

// Digit histograms of the compacted keys (all 8 digits; the slot digits that
// are constant are skipped by the scan's flags).
__global__ void __launch_bounds__(256) k_hist_all(const uint64_t* __restrict__ keys, const RunCtl* rc,
                                                  SortCtl* ctl) {
    __shared__ uint32_t hist[8 * 256];
    for (int j = threadIdx.x; j < 8 * 256; j += blockDim.x) hist[j] = 0;
    __syncthreads();
    const uint64_t n = rc->l_packed & 0xffffffffull;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = keys[i];
#pragma unroll
        for (int p = 0; p < 8; ++p) atomicAdd(&hist[p * 256 + (uint32_t)((k >> (8 * p)) & 255u)], 1u);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < 8 * 256; j += blockDim.x) {
        const uint32_t v = hist[j];
        if (v) atomicAdd(&ctl->hist[j >> 8][j & 255], v);
    }
}

// The sorted compacted points into place: position c of the sorted array holds
// the point that sat at compacted position c0 (its value) of run `slot`.
__global__ void __launch_bounds__(256) k_long_put(const uint64_t* __restrict__ ckeys,
                                                  const uint32_t* __restrict__ cvals,
                                                  const LongRun* __restrict__ runs, const RunCtl* rc,
                                                  const uint32_t* __restrict__ hi, const uint64_t* __restrict__ pv,
                                                  const double* __restrict__ xyz, uint64_t* __restrict__ keys_out,
                                                  uint32_t* __restrict__ perm_out, double* __restrict__ xs,
                                                  double* __restrict__ ys, double* __restrict__ zs) {
    const uint64_t n = rc->l_packed & 0xffffffffull;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
        const LongRun lr = runs[(uint32_t)(ckeys[c] >> 32)];
        const uint64_t i = (uint64_t)lr.start + (cvals[c] - lr.off);  // where the point sat after the passes
        put_sorted((uint64_t)lr.start + (c - lr.off), hi[i], pv[i], xyz, keys_out, perm_out, xs, ys, zs);
    }
}

// The split sort's arrays in input order (no upper-digit pass ran): the upper
// halves, and lower half << 32 | input position.
__global__ void k_pack_iota(const uint64_t* __restrict__ keys, uint32_t* __restrict__ hi, uint64_t* __restrict__ pv,
                            uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        hi[i] = (uint32_t)(keys[i] >> 32);
        pv[i] = (keys[i] << 32) | i;
    }
}

__global__ void k_iota(uint32_t* perm, uint64_t n) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) perm[i] = (uint32_t)i;
}

__global__ void k_gather(const double* __restrict__ xyz, const uint32_t* __restrict__ perm, uint64_t n,
                         double* __restrict__ xs, double* __restrict__ ys, double* __restrict__ zs) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint64_t j = perm[i];
        if (j >= n) j = 0;  // a permutation never does this; guards a failed sort
        xs[i] = xyz[3 * j];
        ys[i] = xyz[3 * j + 1];
        zs[i] = xyz[3 * j + 2];
    }
}

int sm_count(int device) {
    static int cached[64] = {0};
    if (device >= 0 && device < 64 && cached[device]) return cached[device];
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    if (device >= 0 && device < 64) cached[device] = v;
    return v;
}

size_t onesweep_smem() {
    return (size_t)kSortTile * 8 + (size_t)kSortTile * 4 + (size_t)kSortWarps * 256 * 4 + 256 * 4 + 256 * 8;
}

}  // namespace

// Resident k_bbox blocks per SM: its grid is one full wave (with 4 blocks per
// SM asked and 3 resident, the partial second wave cost 116 against 89 us on
// 10M points).
int bbox_blocks_per_sm() {
    static int per = 0;
    if (per == 0) {
        int v = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_bbox, kBboxThreads, 0) != cudaSuccess || v < 1) v = 1;
        per = v;
    }
    return per;
}

cudaError_t launch_bbox_encode(Cloud& c, const double* d_xyz, bool upper_hist_only) {
    cudaError_t e;
    const uint64_t n = c.n;
    const int sms = sm_count(c.device);
    const int grid_bbox = sms * bbox_blocks_per_sm();
    if ((e = c.d_box.reserve(sizeof(BoxGeom))) != cudaSuccess) return e;
    if ((e = c.d_ctl.reserve(sizeof(SortCtl))) != cudaSuccess) return e;
    if ((e = c.parts.reserve(sizeof(double) * 6 * grid_bbox + 64)) != cudaSuccess) return e;
    if ((e = c.keys.reserve(8 * (n ? n : 1))) != cudaSuccess) return e;
    SortCtl* ctl = c.d_ctl.as<SortCtl>();
    if ((e = cudaMemsetAsync(ctl, 0, sizeof(SortCtl), c.stream)) != cudaSuccess) return e;
    k_bbox<<<grid_bbox, kBboxThreads, 0, c.stream>>>(d_xyz, n, c.parts.as<double>(), &ctl->bbox_ctr,
                                                     c.d_box.as<BoxGeom>());
    if (n) {
        const uint64_t want = (n / 2 + kEncThreads) / kEncThreads;
        const int grid = (int)(want < (uint64_t)sms * kEncGridPerSM ? want : (uint64_t)sms * kEncGridPerSM);
        const bool hil = c.params.encoder == OCT_ENC_HILBERT_3D;
        BoxGeom* bg = c.d_box.as<BoxGeom>();
        uint64_t* keys = c.keys.as<uint64_t>();
        if (!upper_hist_only && hil) k_encode<5><<<grid, kEncThreads, 0, c.stream>>>(d_xyz, n, bg, keys, ctl);
        else if (!upper_hist_only) k_encode<1><<<grid, kEncThreads, 0, c.stream>>>(d_xyz, n, bg, keys, ctl);
        else if (hil) k_encode<5, false><<<grid, kEncThreads, 0, c.stream>>>(d_xyz, n, bg, keys, ctl);
        else k_encode<1, false><<<grid, kEncThreads, 0, c.stream>>>(d_xyz, n, bg, keys, ctl);
        k_scan_hist<<<1, 256, 0, c.stream>>>(ctl, n);
    }
    return cudaGetLastError();
}

cudaError_t launch_sort_passes(Cloud& c, const uint32_t skip[8], int* final_sel) {
    cudaError_t e;
    const uint64_t n = c.n;
    *final_sel = 0;
    if ((e = c.perm.reserve(4 * (n ? n : 1))) != cudaSuccess) return e;
    if (n == 0) return cudaSuccess;
    if ((e = c.keys_alt.reserve(8 * n)) != cudaSuccess) return e;
    if ((e = c.perm_alt.reserve(4 * n)) != cudaSuccess) return e;
    const uint64_t tiles = (n + kSortTile - 1) / kSortTile;
    const size_t status_bytes = tiles * 256 * sizeof(unsigned long long);
    if (status_bytes > c.sort_status.bytes) {
        if ((e = c.sort_status.reserve(status_bytes)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(c.sort_status.ptr, 0, c.sort_status.bytes, c.stream)) != cudaSuccess) return e;
        c.sort_epoch = 0;
    }
    // the shared-memory limit is an attribute of the current device's copy of the kernel: set it on every call
    // (cheap, host side), so that clouds on any device and from any host thread launch with it
    const size_t smem = onesweep_smem();
    if ((e = prepare_sort_dyn()) != cudaSuccess) return e;
    DevBuf* kb[2] = {&c.keys, &c.keys_alt};
    DevBuf* vb[2] = {&c.perm, &c.perm_alt};
    int sel = 0;
    bool first = true;
    SortCtl* ctl = c.d_ctl.as<SortCtl>();
    for (int p = 0; p < 8; ++p) {
        if (skip[p]) continue;
        c.sort_epoch = (c.sort_epoch + 1) & ((1u << 22) - 1);
        if (c.sort_epoch == 0) {  // epoch wrapped: clear stale words
            if ((e = cudaMemsetAsync(c.sort_status.ptr, 0, c.sort_status.bytes, c.stream)) != cudaSuccess) return e;
            c.sort_epoch = 1;
        }
        const uint64_t* kin = kb[sel]->as<uint64_t>();
        uint64_t* kout = kb[sel ^ 1]->as<uint64_t>();
        const uint32_t* vin = vb[sel]->as<uint32_t>();
        uint32_t* vout = vb[sel ^ 1]->as<uint32_t>();
        if (first)
            k_onesweep<true, uint64_t, uint32_t><<<(unsigned)tiles, kSortThreads, smem, c.stream>>>(
                kin, nullptr, kout, vout, n, p, ctl, c.sort_status.as<unsigned long long>(), c.sort_epoch,
                c.d_err.as<uint32_t>());
        else
            k_onesweep<false, uint64_t, uint32_t><<<(unsigned)tiles, kSortThreads, smem, c.stream>>>(
                kin, vin, kout, vout, n, p, ctl, c.sort_status.as<unsigned long long>(), c.sort_epoch,
                c.d_err.as<uint32_t>());
        first = false;
        sel ^= 1;
    }
    if (first) {  // every digit constant: the order is the input order
        k_iota<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(c.perm.as<uint32_t>(), n);
        sel = 0;
    }
    *final_sel = sel;
    return cudaGetLastError();
}

// The split sort (upper halves, then runs): the sorted keys go to c.keys_alt,
// the permutation to c.perm, the sorted coordinates to xs / ys / zs.  The
// passes carry each key's lower half with its input position (one 64-bit
// value), so the runs read them in order instead of gathering keys.  When
// RunCtl::big is set (d_run_ctl), runs longer than kRunMid were listed and
// their points are not written yet: launch_sort_long places them.
cudaError_t launch_sort_split(Cloud& c, const uint32_t skip[8], const double* d_xyz, int* out_sel) {
    cudaError_t e;
    const uint64_t n = c.n;
    *out_sel = 0;
    const size_t nn = n ? n : 1;
    if ((e = c.keys_alt.reserve(8 * nn)) != cudaSuccess) return e;
    if ((e = c.perm.reserve(4 * nn)) != cudaSuccess) return e;
    if ((e = c.keys_hi.reserve(4 * nn)) != cudaSuccess) return e;
    if ((e = c.keys_hi_alt.reserve(4 * nn)) != cudaSuccess) return e;
    if ((e = c.run_pv.reserve(8 * nn)) != cudaSuccess) return e;
    if ((e = c.run_pv_alt.reserve(8 * nn)) != cudaSuccess) return e;
    if ((e = c.run_ctl.reserve(sizeof(RunCtl))) != cudaSuccess) return e;
    if ((e = c.run_list.reserve(8 * (n / (kRunSmall + 1) + 1))) != cudaSuccess) return e;
    if ((e = c.run_long.reserve(sizeof(LongRun) * (n / (kRunMid + 1) + 1))) != cudaSuccess) return e;
    if ((e = c.xs.reserve(8 * nn)) != cudaSuccess) return e;
    if ((e = c.ys.reserve(8 * nn)) != cudaSuccess) return e;
    if ((e = c.zs.reserve(8 * nn)) != cudaSuccess) return e;
    RunCtl* rc = c.run_ctl.as<RunCtl>();
    RunCtl rc0{};
    rc0.cap = (uint32_t)(n / (kRunSmall + 1) + 1);
    if ((e = cudaMemcpyAsync(rc, &rc0, sizeof(RunCtl), cudaMemcpyHostToDevice, c.stream)) != cudaSuccess) return e;
    if (n == 0) return cudaSuccess;
    const uint64_t tiles = (n + kSortTile - 1) / kSortTile;
    const size_t status_bytes = tiles * 256 * sizeof(unsigned long long);
    if (status_bytes > c.sort_status.bytes) {
        if ((e = c.sort_status.reserve(status_bytes)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(c.sort_status.ptr, 0, c.sort_status.bytes, c.stream)) != cudaSuccess) return e;
        c.sort_epoch = 0;
    }
    // 32-bit keys with 64-bit values: the same 12 bytes per tile slot as the 8-pass sort's
    const size_t smem = onesweep_smem();
    if ((e = cudaFuncSetAttribute(k_onesweep<true, uint32_t, uint64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_onesweep<false, uint32_t, uint64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem)) != cudaSuccess)
        return e;
    DevBuf* kb[2] = {&c.keys_hi, &c.keys_hi_alt};
    DevBuf* vb[2] = {&c.run_pv, &c.run_pv_alt};
    int sel = 0;
    bool first = true;
    SortCtl* ctl = c.d_ctl.as<SortCtl>();
    for (int p = 4; p < 8; ++p) {  // the digits of the upper halves
        if (skip[p]) continue;
        c.sort_epoch = (c.sort_epoch + 1) & ((1u << 22) - 1);
        if (c.sort_epoch == 0) {
            if ((e = cudaMemsetAsync(c.sort_status.ptr, 0, c.sort_status.bytes, c.stream)) != cudaSuccess) return e;
            c.sort_epoch = 1;
        }
        const uint32_t* kin = kb[sel]->as<uint32_t>();
        uint32_t* kout = kb[sel ^ 1]->as<uint32_t>();
        const uint64_t* vin = vb[sel]->as<uint64_t>();
        uint64_t* vout = vb[sel ^ 1]->as<uint64_t>();
        if (first)
            k_onesweep<true, uint32_t, uint64_t><<<(unsigned)tiles, kSortThreads, smem, c.stream>>>(
                nullptr, nullptr, kout, vout, n, p, ctl, c.sort_status.as<unsigned long long>(), c.sort_epoch,
                c.d_err.as<uint32_t>(), nullptr, nullptr, c.keys.as<uint64_t>());
        else
            k_onesweep<false, uint32_t, uint64_t><<<(unsigned)tiles, kSortThreads, smem, c.stream>>>(
                kin, vin, kout, vout, n, p, ctl, c.sort_status.as<unsigned long long>(), c.sort_epoch,
                c.d_err.as<uint32_t>());
        first = false;
        sel ^= 1;
    }
    const int sms = sm_count(c.device);
    const uint64_t want = (n + 255) / 256;
    const int grid = (int)(want < (uint64_t)sms * 8 ? want : (uint64_t)sms * 8);
    if (first) {  // every upper digit constant: one run in input order
        k_pack_iota<<<grid, 256, 0, c.stream>>>(c.keys.as<uint64_t>(), c.keys_hi.as<uint32_t>(),
                                                 c.run_pv.as<uint64_t>(), n);
        sel = 0;
    }
    c.split_sel = sel;  // the upper halves and payloads the runs read (and the long-run stage)
    const uint32_t* hi = kb[sel]->as<uint32_t>();
    const uint64_t* pv = vb[sel]->as<uint64_t>();
    uint32_t* perm_out = c.perm.as<uint32_t>();
    k_runs_small<<<grid, 256, 0, c.stream>>>(hi, pv, d_xyz, n, c.keys_alt.as<uint64_t>(), perm_out, c.xs.as<double>(),
                                            c.ys.as<double>(), c.zs.as<double>(), rc, c.run_list.as<uint32_t>(),
                                            c.run_long.as<LongRun>());
    k_runs_warp<<<sms * 8, kRunWarpThreads, 0, c.stream>>>(hi, pv, d_xyz, c.keys_alt.as<uint64_t>(), perm_out,
                                                           c.xs.as<double>(), c.ys.as<double>(), c.zs.as<double>(),
                                                           rc, c.run_list.as<uint32_t>());
    k_runs_mid<<<sms * 4, kRunMidThreads, 0, c.stream>>>(hi, pv, d_xyz, c.keys_alt.as<uint64_t>(), perm_out,
                                                     c.xs.as<double>(), c.ys.as<double>(), c.zs.as<double>(), rc,
                                                     c.run_list.as<uint32_t>());
    return cudaGetLastError();
}

// The split sort's long runs (after launch_sort_split, when RunCtl::big is set;
// l_count runs, l_total points, as RunCtl::l_packed holds them): compact their points
// keyed by (run slot, lower key half), sort them with 4 + (slot bytes) onesweep
// passes, put them in place.  The compacted keys use c.keys (the encode's keys,
// not read again) and c.run_pv_alt, the values c.perm_alt and c.keys_hi_alt.
cudaError_t launch_sort_long(Cloud& c, const double* d_xyz, uint32_t l_count, uint32_t l_total) {
    cudaError_t e;
    const uint64_t T = l_total;
    if (l_count == 0 || T == 0) return cudaSuccess;
    if ((e = c.keys.reserve(8 * T)) != cudaSuccess) return e;
    if ((e = c.run_pv_alt.reserve(8 * T)) != cudaSuccess) return e;
    if ((e = c.perm_alt.reserve(4 * T)) != cudaSuccess) return e;
    if ((e = c.keys_hi_alt.reserve(4 * T)) != cudaSuccess) return e;
    const uint64_t tiles = (T + kSortTile - 1) / kSortTile;
    const size_t status_bytes = tiles * 256 * sizeof(unsigned long long);
    if (status_bytes > c.sort_status.bytes) {
        if ((e = c.sort_status.reserve(status_bytes)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(c.sort_status.ptr, 0, c.sort_status.bytes, c.stream)) != cudaSuccess) return e;
        c.sort_epoch = 0;
    }
    const size_t smem = onesweep_smem();
    if ((e = prepare_sort_dyn()) != cudaSuccess) return e;
    const RunCtl* rc = c.run_ctl.as<RunCtl>();
    const LongRun* runs = c.run_long.as<LongRun>();
    DevBuf* hb[2] = {&c.keys_hi, &c.keys_hi_alt};
    DevBuf* pb[2] = {&c.run_pv, &c.run_pv_alt};
    const uint32_t* hi = hb[c.split_sel]->as<uint32_t>();
    const uint64_t* pv = pb[c.split_sel]->as<uint64_t>();
    if (c.split_sel != 0) return cudaErrorInvalidValue;  // the split sort always ends in its first buffers
    SortCtl* ctl = c.d_ctl.as<SortCtl>();
    if ((e = cudaMemsetAsync(ctl, 0, sizeof(SortCtl), c.stream)) != cudaSuccess) return e;
    const int sms = sm_count(c.device);
    DevBuf* kb[2] = {&c.keys, &c.run_pv_alt};
    DevBuf* vb[2] = {&c.perm_alt, &c.keys_hi_alt};
    k_long_compact<<<(unsigned)(l_count < (uint32_t)sms * 8 ? l_count : (uint32_t)sms * 8), 256, 0, c.stream>>>(
        pv, runs, rc, kb[0]->as<uint64_t>());
    const uint64_t want = (T + 255) / 256;
    const int grid = (int)(want < (uint64_t)sms * 4 ? want : (uint64_t)sms * 4);
    k_hist_all<<<grid, 256, 0, c.stream>>>(kb[0]->as<uint64_t>(), rc, ctl);
    k_scan_hist<<<1, 256, 0, c.stream>>>(ctl, T);
    int slot_bytes = 0;
    for (uint32_t v = l_count - 1; v; v >>= 8) ++slot_bytes;
    int sel = 0;
    for (int p = 0; p < 4 + slot_bytes; ++p) {
        c.sort_epoch = (c.sort_epoch + 1) & ((1u << 22) - 1);
        if (c.sort_epoch == 0) {
            if ((e = cudaMemsetAsync(c.sort_status.ptr, 0, c.sort_status.bytes, c.stream)) != cudaSuccess) return e;
            c.sort_epoch = 1;
        }
        const uint64_t* kin = kb[sel]->as<uint64_t>();
        uint64_t* kout = kb[sel ^ 1]->as<uint64_t>();
        const uint32_t* vin = vb[sel]->as<uint32_t>();
        uint32_t* vout = vb[sel ^ 1]->as<uint32_t>();
        if (p == 0)
            k_onesweep<true, uint64_t, uint32_t><<<(unsigned)tiles, kSortThreads, smem, c.stream>>>(
                kin, nullptr, kout, vout, T, p, ctl, c.sort_status.as<unsigned long long>(), c.sort_epoch,
                c.d_err.as<uint32_t>());
        else
            k_onesweep<false, uint64_t, uint32_t><<<(unsigned)tiles, kSortThreads, smem, c.stream>>>(
                kin, vin, kout, vout, T, p, ctl, c.sort_status.as<unsigned long long>(), c.sort_epoch,
                c.d_err.as<uint32_t>());
        sel ^= 1;
    }
    k_long_put<<<grid, 256, 0, c.stream>>>(kb[sel]->as<uint64_t>(), vb[sel]->as<uint32_t>(), runs, rc, hi, pv, d_xyz,
                                           c.keys_alt.as<uint64_t>(), c.perm.as<uint32_t>(), c.xs.as<double>(),
                                           c.ys.as<double>(), c.zs.as<double>());
    return cudaGetLastError();
}

cudaError_t launch_gather(Cloud& c, const double* d_xyz, const uint32_t* d_perm, int /*sel*/) {
    cudaError_t e;
    const uint64_t n = c.n;
    const size_t b = 8 * (n ? n : 1);
    if ((e = c.xs.reserve(b)) != cudaSuccess) return e;
    if ((e = c.ys.reserve(b)) != cudaSuccess) return e;
    if ((e = c.zs.reserve(b)) != cudaSuccess) return e;
    if (n == 0) return cudaSuccess;
    const int sms = sm_count(c.device);
    const uint64_t want = (n + 255) / 256;
    const int grid = (int)(want < (uint64_t)sms * 8 ? want : (uint64_t)sms * 8);
    k_gather<<<grid, 256, 0, c.stream>>>(d_xyz, d_perm, n, c.xs.as<double>(), c.ys.as<double>(),
                                         c.zs.as<double>());
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Query ordering for the packet searches: the query centres are keyed with the
// cloud's box and curve and stably sorted by the top 24 key bits (3 onesweep
// passes), so that the 32 queries of a warp are spatial neighbours.
// ---------------------------------------------------------------------------
// Device-sized sort of a batch's query keys (the batched engine): the key
// count and the epoch base are read on the device, and every pass runs a fixed
// persistent grid, so the launch sequence can be captured once as a graph.

cudaError_t prepare_sort_dyn() {
    const int smem = (int)onesweep_smem();
    cudaError_t e = cudaFuncSetAttribute(k_onesweep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_onesweep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

size_t sort_tile_keys() { return kSortTile; }

cudaError_t launch_sort_dyn(int device, cudaStream_t s, uint64_t* k0, uint64_t* k1, uint32_t* v0, uint32_t* v1,
                            const uint64_t* d_n, uint64_t max_n, int passes, SortCtl* ctl,
                            unsigned long long* status, const uint32_t* d_epoch, uint32_t* err,
                            uint32_t** result_vals) {
    const size_t smem = onesweep_smem();
    const uint64_t max_tiles = (max_n + kSortTile - 1) / kSortTile;
    const uint64_t resident = (uint64_t)sm_count(device) * kSortBlocksPerSM;
    const unsigned grid = (unsigned)(max_tiles < resident ? (max_tiles ? max_tiles : 1) : resident);
    k_scan_hist<<<1, 256, 0, s>>>(ctl, 0, d_n);
    uint64_t* kb[2] = {k0, k1};
    uint32_t* vb[2] = {v0, v1};
    for (int p = 0; p < passes; ++p) {
        const int i = p & 1, o = i ^ 1;
        if (p == 0)
            k_onesweep<true, uint64_t, uint32_t><<<grid, kSortThreads, smem, s>>>(
                kb[i], nullptr, kb[o], vb[o], 0, p, ctl, status, 0, err, d_n, d_epoch);
        else
            k_onesweep<false, uint64_t, uint32_t><<<grid, kSortThreads, smem, s>>>(
                kb[i], vb[i], kb[o], vb[o], 0, p, ctl, status, 0, err, d_n, d_epoch);
    }
    *result_vals = vb[passes & 1];
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------

namespace {

template <int ENC>
__global__ void __launch_bounds__(kEncThreads) k_query_keys(const double* __restrict__ q, uint64_t nq,
                                                            const BoxGeom* __restrict__ bg,
                                                            uint64_t* __restrict__ keys, SortCtl* ctl) {
    __shared__ uint32_t hist[3 * 256];
    for (int j = threadIdx.x; j < 3 * 256; j += blockDim.x) hist[j] = 0;
    const double c0 = bg->box.center[0], c1 = bg->box.center[1], c2 = bg->box.center[2];
    const double r0 = bg->box.radii[0], r1 = bg->box.radii[1], r2 = bg->box.radii[2];
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += stride) {
        const uint64_t k = sfc_encode<ENC>(anchor_coord(q[3 * i], c0, r0), anchor_coord(q[3 * i + 1], c1, r1),
                                           anchor_coord(q[3 * i + 2], c2, r2));
        keys[i] = k;
#pragma unroll
        for (int p = 5; p < 8; ++p) atomicAdd(&hist[(p - 5) * 256 + (uint32_t)((k >> (8 * p)) & 255u)], 1u);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < 3 * 256; j += blockDim.x) {
        const uint32_t v = hist[j];
        if (v) atomicAdd(&ctl->hist[5 + (j >> 8)][j & 255], v);
    }
}

}  // namespace

cudaError_t launch_query_order(Cloud& c, const double* d_centers, uint64_t nq, const uint32_t** d_order) {
    cudaError_t e;
    *d_order = nullptr;
    if (nq == 0) return cudaSuccess;
    const uint64_t tiles = (nq + kSortTile - 1) / kSortTile;
    if ((e = c.qs_keys.reserve(8 * nq)) != cudaSuccess) return e;
    if ((e = c.qs_keys_alt.reserve(8 * nq)) != cudaSuccess) return e;
    if ((e = c.qs_ord.reserve(4 * nq)) != cudaSuccess) return e;
    if ((e = c.qs_ord_alt.reserve(4 * nq)) != cudaSuccess) return e;
    if ((e = c.qs_ctl.reserve(sizeof(SortCtl))) != cudaSuccess) return e;
    const size_t status_bytes = tiles * 256 * sizeof(unsigned long long);
    if (status_bytes > c.qs_status.bytes) {
        if ((e = c.qs_status.reserve(status_bytes)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(c.qs_status.ptr, 0, c.qs_status.bytes, c.stream)) != cudaSuccess) return e;
        c.qs_epoch = 0;
    }
    const size_t smem = onesweep_smem();
    if ((e = prepare_sort_dyn()) != cudaSuccess) return e;
    SortCtl* ctl = c.qs_ctl.as<SortCtl>();
    if ((e = cudaMemsetAsync(ctl, 0, sizeof(SortCtl), c.stream)) != cudaSuccess) return e;
    const int sms = sm_count(c.device);
    const uint64_t want = (nq + kEncThreads - 1) / kEncThreads;
    const int grid = (int)(want < (uint64_t)sms * kEncGridPerSM ? want : (uint64_t)sms * kEncGridPerSM);
    const BoxGeom* bg = c.d_box.as<BoxGeom>();
    if (c.params.encoder == OCT_ENC_HILBERT_3D)
        k_query_keys<5><<<grid, kEncThreads, 0, c.stream>>>(d_centers, nq, bg, c.qs_keys.as<uint64_t>(), ctl);
    else
        k_query_keys<1><<<grid, kEncThreads, 0, c.stream>>>(d_centers, nq, bg, c.qs_keys.as<uint64_t>(), ctl);
    k_scan_hist<<<1, 256, 0, c.stream>>>(ctl, nq);
    DevBuf* kb[2] = {&c.qs_keys, &c.qs_keys_alt};
    DevBuf* vb[2] = {&c.qs_ord, &c.qs_ord_alt};
    int sel = 0;
    for (int p = 5; p < 8; ++p) {
        c.qs_epoch = (c.qs_epoch + 1) & ((1u << 22) - 1);
        if (c.qs_epoch == 0) {
            if ((e = cudaMemsetAsync(c.qs_status.ptr, 0, c.qs_status.bytes, c.stream)) != cudaSuccess) return e;
            c.qs_epoch = 1;
        }
        if (p == 5)
            k_onesweep<true, uint64_t, uint32_t><<<(unsigned)tiles, kSortThreads, smem, c.stream>>>(
                kb[sel]->as<uint64_t>(), nullptr, kb[sel ^ 1]->as<uint64_t>(), vb[sel ^ 1]->as<uint32_t>(), nq, p,
                ctl, c.qs_status.as<unsigned long long>(), c.qs_epoch, c.d_err.as<uint32_t>());
        else
            k_onesweep<false, uint64_t, uint32_t><<<(unsigned)tiles, kSortThreads, smem, c.stream>>>(
                kb[sel]->as<uint64_t>(), vb[sel]->as<uint32_t>(), kb[sel ^ 1]->as<uint64_t>(),
                vb[sel ^ 1]->as<uint32_t>(), nq, p, ctl, c.qs_status.as<unsigned long long>(), c.qs_epoch,
                c.d_err.as<uint32_t>());
        sel ^= 1;
    }
    *d_order = vb[sel]->as<uint32_t>();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free encode + sort (oct_encode_sort_noalloc).
//
// For callers that cannot allocate device memory at call time: code that runs
// inside a memory pool or allocator it does not own, a plugin host that
// forbids cudaMalloc/cudaFree on its streams, or a real-time loop that must
// not block on the allocator (cudaMalloc/cudaFree synchronise the device).
// The caller passes device buffers for the points and every output; the
// scratch the sort needs (second key/id buffer, look-back words, histograms,
// bounding-box partials) lives in the fixed array below, which every GPU that
// loads this library holds until the process exits.
// ---------------------------------------------------------------------------

constexpr uint64_t kNoAllocTiles = (OCT_NOALLOC_MAX_POINTS + kSortTile - 1) / kSortTile;
constexpr int kNoAllocBboxGrid = 148 * 4;

struct NoAllocScratch {
    uint64_t keys_alt[OCT_NOALLOC_MAX_POINTS];            // 2 MiB
    uint32_t perm_alt[OCT_NOALLOC_MAX_POINTS];            // 1 MiB
    unsigned long long status[kNoAllocTiles * 256];       // look-back words, 256 per tile
    SortCtl ctl;
    BoxGeom bg;
    double partial[6 * kNoAllocBboxGrid];
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// The Box (center, radii, min, max: the 12 leading doubles of BoxGeom) into
// the caller's buffer.  If a sort pass's bounded look-back gave up (its error
// word is set) some keys and ids were never written; the radii are then set
// to -1.0, a value no Box can hold (radii are half the extent: >= 0 or NaN).
__global__ void k_noalloc_box(const BoxGeom* bg, const uint32_t* err, double* box12) {
    const int i = threadIdx.x;
    if (i >= 12) return;
    const double* src = reinterpret_cast<const double*>(&bg->box);
    box12[i] = (*err != 0u && i >= 3 && i < 6) ? -1.0 : src[i];
}

namespace {

std::mutex g_noalloc_mu;
NoAllocScratch* g_noalloc_ptr[64] = {nullptr};

// Device address of the scratch array on the current device.  The array's
// name is only a host-side stand-in in host code, so the address comes from
// cudaGetSymbolAddress, once per device, with that device current.
int noalloc_setup(int dev, NoAllocScratch** out) {
    if (dev < 0 || dev >= 64) return OCT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return OCT_ERR_CUDA;
        }
        const int smem = (int)onesweep_smem();
        if (cudaFuncSetAttribute(k_onesweep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_onesweep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
                cudaSuccess) {
            cudaGetLastError();
            return OCT_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return OCT_OK;
}

}  // namespace

// A kernel of this file's device code, for preload_kernels.
const void* kernel_anchor_encode_sort() { return reinterpret_cast<const void*>(&k_iota); }

}  // namespace octb

extern "C" int oct_encode_sort_noalloc(int encoder, const double* d_xyz, uint64_t n, uint64_t* d_keys,
                                       uint32_t* d_perm, double* d_box12, void* stream) {
    using namespace octb;
    if (encoder != OCT_ENC_MORTON_3D && encoder != OCT_ENC_HILBERT_3D) return OCT_ERR_INVALID_ARG;
    if (n > OCT_NOALLOC_MAX_POINTS) return OCT_ERR_INVALID_ARG;
    if (n && (!d_xyz || !d_keys || !d_perm)) return OCT_ERR_INVALID_ARG;
    if (!d_box12) return OCT_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return OCT_ERR_NO_DEVICE;
    }
    NoAllocScratch* sc = nullptr;
    int st = noalloc_setup(dev, &sc);
    if (st != OCT_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    SortCtl* ctl = &sc->ctl;
    const uint64_t tiles = (n + kSortTile - 1) / kSortTile;
    // every call shares the scratch: clear what must start at zero
    if (cudaMemsetAsync(ctl, 0, sizeof(SortCtl), s) != cudaSuccess) return OCT_ERR_CUDA;
    if (tiles && cudaMemsetAsync(sc->status, 0, tiles * 256 * sizeof(unsigned long long), s) != cudaSuccess)
        return OCT_ERR_CUDA;
    k_bbox<<<kNoAllocBboxGrid, kBboxThreads, 0, s>>>(d_xyz, n, sc->partial, &ctl->bbox_ctr, &sc->bg);
    if (n) {
        const uint64_t want = (n + kEncThreads - 1) / kEncThreads;
        const int grid = (int)(want < (uint64_t)kNoAllocBboxGrid ? want : (uint64_t)kNoAllocBboxGrid);
        if (encoder == OCT_ENC_HILBERT_3D) k_encode<5><<<grid, kEncThreads, 0, s>>>(d_xyz, n, &sc->bg, d_keys, ctl);
        else k_encode<1><<<grid, kEncThreads, 0, s>>>(d_xyz, n, &sc->bg, d_keys, ctl);
        k_scan_hist<<<1, 256, 0, s>>>(ctl, n);
        // all 8 digit passes (no host readback of the skip flags), so the result
        // ends in the caller's buffers: caller -> scratch -> caller ...
        const size_t smem = onesweep_smem();
        uint32_t* err = reinterpret_cast<uint32_t*>(&ctl->pad);
        for (int p = 0; p < 8; ++p) {
            const bool to_scratch = (p % 2) == 0;
            const uint64_t* kin = to_scratch ? d_keys : sc->keys_alt;
            uint64_t* kout = to_scratch ? sc->keys_alt : d_keys;
            const uint32_t* vin = to_scratch ? d_perm : sc->perm_alt;
            uint32_t* vout = to_scratch ? sc->perm_alt : d_perm;
            if (p == 0)
                k_onesweep<true, uint64_t, uint32_t><<<(unsigned)tiles, kSortThreads, smem, s>>>(
                    kin, nullptr, kout, vout, n, p, ctl, sc->status, (uint32_t)(p + 1), err);
            else
                k_onesweep<false, uint64_t, uint32_t><<<(unsigned)tiles, kSortThreads, smem, s>>>(
                    kin, vin, kout, vout, n, p, ctl, sc->status, (uint32_t)(p + 1), err);
        }
    }
    // Box (center, radii, min, max), radii -1.0 if a look-back gave up
    k_noalloc_box<<<1, 32, 0, s>>>(&sc->bg, reinterpret_cast<const uint32_t*>(&ctl->pad), d_box12);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? OCT_OK : OCT_ERR_CUDA;
}
