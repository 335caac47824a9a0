// Batched multi-cloud search engine (oct_engine_* in include/octree_b200.h).
//
// No reference counterpart: the reference answers one query per OpenMP thread
// per call (neighbor_benchmarks.hpp:502-568 around linear_octree.hpp:746-784
// and 899-942).  Here a batch of requests - radius or kNN centre sets, each
// against one built cloud - runs as one device pass:
//   1. the host packs the requests into a table (SearchReq, grouped by kernel
//      variant) and a descriptor of group sizes (DynGroup), and copies both to
//      the device in one transfer;
//   2. k_batch_keys gives every centre the key (request index, top 24 bits of
//      its curve key in its cloud's frame) and the digit histograms; a 3-5
//      pass onesweep sort of these keys orders every request's centres along
//      its cloud's curve while each request keeps its own position range;
//   3. per radius variant one persistent packet launch counts, a scan turns
//      the counts into CSR offsets and a second launch fills; the kNN groups
//      run at the same time on a forked stream;
//   4. a 16-byte summary (radius total, error word) and the per-request result
//      sizes come back.
// Every size of steps 2-4 is read on the device, so a batch shape (the set of
// variants and the pass count) is captured once as a CUDA graph and replayed
// for every later batch of that shape.  When the radius results outgrow the
// result array the host grows it and runs the batch again.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "cloud.h"
#include "sfc.cuh"

using namespace octb;

namespace {

constexpr int kRadiusVariants = 16;  // kernel (4) x algo (neighbors, prune) x FP32 filter (2)
constexpr int kKnnVariants = 6;      // k <= 32, 64 (register lists), 128, 256, 512, 1024 (shared-memory lists)
constexpr int kGroups = kRadiusVariants + kKnnVariants;
constexpr int kScanBlocks = 296;
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kKeyThreads = 256;
constexpr uint32_t kEpochStep = 8;
constexpr uint32_t kEpochLimit = (1u << 22) - 1;

struct EngineDyn {
    DynGroup groups[kGroups];
    DynGroup fb[2];     // group kNN (k <= 32, 64): the queries handed back to the per-query kernel
    uint64_t n_total;   // query positions of the batch (the sort size)
    uint64_t n_radius;  // radius positions [0, n_radius); kNN positions follow
    uint32_t nreq;      // requests in the table (non-empty ones)
    uint32_t pad;
};

struct Summary {
    unsigned long long radius_total;
    uint32_t err;
    uint32_t pad;
};

// Per request of the table: first result and result count (radius requests).
struct ReqTotal {
    unsigned long long begin;
    unsigned long long count;
};

int radius_variant(int kernel, int algo, int fp32) {
    return (kernel << 2) | ((algo == OCT_NEIGHBORS_PRUNE) ? 2 : 0) | (fp32 ? 1 : 0);
}

__global__ void k_epoch_advance(uint32_t* epoch) { *epoch = (*epoch + kEpochStep) & kEpochLimit; }

// Sort key of every centre: (table index << 24) | top 24 bits of its SFC key
// in its cloud's Box, with the digit histograms of the `passes` low bytes.
__global__ void __launch_bounds__(kKeyThreads) k_batch_keys(const EngineDyn* __restrict__ dyn,
                                                            const SearchReq* __restrict__ table,
                                                            uint64_t* __restrict__ keys, SortCtl* ctl, int passes) {
    __shared__ uint32_t hist[5 * 256];
    for (int j = threadIdx.x; j < 5 * 256; j += blockDim.x) hist[j] = 0;
    __syncthreads();
    const uint64_t n = dyn->n_total;
    const uint32_t nreq = dyn->nreq;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint32_t lo = 0, hi = nreq;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (table[mid].q_begin <= i) lo = mid;
            else hi = mid;
        }
        const SearchReq& rq = table[lo];
        const double* c = rq.centers + 3 * (i - rq.q_begin);
        const BoxD* b = rq.cv.box;
        const uint32_t ax = anchor_coord(c[0], b->center[0], b->radii[0]);
        const uint32_t ay = anchor_coord(c[1], b->center[1], b->radii[1]);
        const uint32_t az = anchor_coord(c[2], b->center[2], b->radii[2]);
        const uint64_t code =
            rq.cv.encoder == OCT_ENC_HILBERT_3D ? sfc_encode<5>(ax, ay, az) : sfc_encode<1>(ax, ay, az);
        const uint64_t key = ((uint64_t)lo << 24) | (code >> 39);
        keys[i] = key;
        for (int p = 0; p < passes; ++p) atomicAdd(&hist[p * 256 + (uint32_t)((key >> (8 * p)) & 255u)], 1u);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < passes * 256; j += blockDim.x) {
        const uint32_t v = hist[j];
        if (v) atomicAdd(&ctl->hist[j >> 8][j & 255], v);
    }
}

__device__ __forceinline__ unsigned long long block_excl_scan_u64(unsigned long long v, unsigned long long* tot) {
    __shared__ unsigned long long wsum[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    unsigned long long pre = 0, all = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) {
        if (w < warp) pre += wsum[w];
        all += wsum[w];
    }
    __syncthreads();
    *tot = all;
    return pre + x - v;
}

// Scan of the radius counts [0, n) with n read on the device: fixed grid,
// block b owns a contiguous chunk.
__global__ void __launch_bounds__(kScanThreads) k_escan_reduce(const unsigned long long* __restrict__ in,
                                                               const uint64_t* d_n, unsigned long long* part) {
    const uint64_t n = *d_n;
    const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t b = (uint64_t)blockIdx.x * chunk, e = (b + chunk < n) ? b + chunk : n;
    unsigned long long s = 0;
    for (uint64_t i = b + threadIdx.x; i < e; i += kScanThreads) s += in[i];
    unsigned long long tot;
    block_excl_scan_u64(s, &tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads) k_escan_top(unsigned long long* part, int m, Summary* sum) {
    unsigned long long carry = 0;
    for (int b = 0; b < m; b += kScanThreads) {
        const int i = b + threadIdx.x;
        const unsigned long long v = (i < m) ? part[i] : 0ull;
        unsigned long long tot;
        const unsigned long long x = block_excl_scan_u64(v, &tot);
        if (i < m) part[i] = carry + x;
        carry += tot;
    }
    if (threadIdx.x == 0) {
        part[m] = carry;
        sum->radius_total = carry;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_escan_apply(const unsigned long long* __restrict__ in,
                                                              const uint64_t* d_n,
                                                              const unsigned long long* __restrict__ part,
                                                              unsigned long long* __restrict__ out) {
    const uint64_t n = *d_n;
    const uint64_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t b = (uint64_t)blockIdx.x * chunk, e = (b + chunk < n) ? b + chunk : n;
    unsigned long long carry = part[blockIdx.x];
    constexpr int kTile = kScanThreads * kScanItems;
    for (uint64_t t = b; t < e; t += kTile) {
        unsigned long long v[kScanItems];
        unsigned long long s = 0;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            const uint64_t i = t + (uint64_t)threadIdx.x * kScanItems + j;
            v[j] = (i < e) ? in[i] : 0ull;
            s += v[j];
        }
        unsigned long long tot;
        unsigned long long x = carry + block_excl_scan_u64(s, &tot);
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            const uint64_t i = t + (uint64_t)threadIdx.x * kScanItems + j;
            if (i < e) out[i] = x;
            x += v[j];
        }
        carry += tot;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = part[gridDim.x];
}

// First result and result count of every radius request of the table.
__global__ void k_req_totals(const EngineDyn* __restrict__ dyn, const SearchReq* __restrict__ table,
                             const unsigned long long* __restrict__ offs, ReqTotal* __restrict__ tot) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= dyn->nreq) return;
    const SearchReq& q = table[r];
    if (q.q_end <= dyn->n_radius) {
        tot[r].begin = offs[q.q_begin];
        tot[r].count = offs[q.q_end] - offs[q.q_begin];
    } else {
        tot[r].begin = 0;
        tot[r].count = 0;
    }
}

// One warp per centre of a radius request: its neighbour count and the sum of
// mix64 over its neighbours (the CSR offsets are the batch's, not rebased).
__global__ void __launch_bounds__(256) k_csr_hash(const unsigned long long* __restrict__ offs,
                                                  const uint32_t* __restrict__ out, uint64_t nq,
                                                  unsigned long long* __restrict__ counts,
                                                  unsigned long long* __restrict__ hashes) {
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t q = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < nq; q += nwarps) {
        const unsigned long long b = offs[q], e = offs[q + 1];
        unsigned long long h = 0;
        for (unsigned long long j = b + lane; j < e; j += 32) h += mix64(out[j]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) h += __shfl_xor_sync(0xffffffffu, h, off);
        if (lane == 0) {
            counts[q] = e - b;
            hashes[q] = h;
        }
    }
}

__global__ void k_rebase(const unsigned long long* __restrict__ in, uint64_t n, unsigned long long* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i] - in[0];
}

int sm_count_e(int device) {
    int v = 148;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v;
}

struct DeviceGuardE {
    int prev = -1;
    explicit DeviceGuardE(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuardE() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

namespace octb {
// A kernel of this file's device code, for preload_kernels.
const void* kernel_anchor_engine() { return reinterpret_cast<const void*>(&k_epoch_advance); }
}  // namespace octb

struct oct_engine_s {
    int device = 0;
    uint32_t flags = 0;
    int sms = 148;
    cudaStream_t stream = nullptr, side = nullptr;
    bool own_stream = false;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    std::string last_error;
    // configuration (oct_engine_set_config / autotune)
    int fp32 = 0;
    uint32_t bucket = 128;
    int radius_bps = 0, knn_bps = 0;
    int serial = 0;  // 1: kNN after the radius search on one stream; 0: kNN forked beside it
    int knn_group = 1;  // kNN with k <= 64: groups of kKnnGroupQueries queries per warp (0: one per warp)
    // device arrays
    DevBuf desc;  // EngineDyn, then the SearchReq table
    DevBuf keys[2], ord[2];
    DevBuf sort_ctl, sort_status, epoch;
    DevBuf counts, offs, part, out;
    DevBuf knn_idx, knn_d2, knn_counts;
    DevBuf ctrs, stats, summary, totals;
    DevBuf ck_pool, ck_next, ck_first, ck_ctr;  // one-pass radius: result chunks (ck_next has one word per chunk)
    DevBuf knn_fb;  // group kNN fallback list, one entry per query position
    DevBuf knn_heads;  // group kNN: the heads' largest k-th distances (f64 per head)
    DevBuf hash_out;   // oct_engine_copy_radius_hash's counts and hashes before they go to the host
    // the growable device arrays above come from this pool in stream order (cudaMallocFromPoolAsync /
    // cudaFreeAsync on `stream`), so growing one never waits for the device: with batches of other engines
    // running, a cudaFree / cudaMalloc would wait for all of them
    cudaMemPool_t pool = nullptr;
    // pinned host staging
    unsigned char* h_stage = nullptr;
    size_t h_stage_bytes = 0;
    Summary* h_summary = nullptr;
    ReqTotal* h_totals = nullptr;
    size_t h_totals_cap = 0;
    uint32_t host_epoch = 0;
    struct Graph {
        uint64_t sig;
        bool one_cloud;
        CloudView view;  // the cloud a one-cloud graph's kernels take as parameters
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;
    bool one_cloud = false;  // every request of the current batch is on one cloud
    CloudView one_view{};
    // the batch in flight (or the last one)
    bool in_flight = false;
    bool have_results = false;
    uint64_t sig = 0;
    int passes = 3;
    uint64_t n_total = 0, n_radius = 0, knn_slots = 0;
    uint32_t nreq = 0;
    size_t desc_bytes = 0;
    uint64_t radius_total = 0;
    float last_ms = 0.f;
    std::vector<oct_request_place> places;  // per request of the caller
    std::vector<int32_t> place_row;         // table row of each caller request, -1 if empty
    std::vector<int32_t> place_type;
};

namespace {

int fail(oct_engine e, int status, const std::string& msg) {
    e->last_error = msg;
    return status;
}

int cuda_fail_e(oct_engine e, cudaError_t err, const char* what) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s: %s (%s)", what, cudaGetErrorName(err), cudaGetErrorString(err));
    cudaGetLastError();
    return fail(e, err == cudaErrorMemoryAllocation ? OCT_ERR_OUT_OF_MEMORY : OCT_ERR_CUDA, buf);
}

#define EK(expr)                                                  \
    do {                                                          \
        cudaError_t _e = (expr);                                  \
        if (_e != cudaSuccess) return cuda_fail_e(e, _e, #expr);  \
    } while (0)

void drop_graphs(oct_engine e) {
    for (auto& g : e->graphs) cudaGraphExecDestroy(g.exec);
    e->graphs.clear();
}

// Grow a device array (by half again at least); a new address drops the
// captured graphs, whose nodes hold the old one.
// A growable array of the engine: the old storage is freed and the new one
// taken from the engine's pool in the engine stream's order (every earlier use
// of the old storage is on that stream, or joined into it).
int grow(oct_engine e, DevBuf& b, size_t bytes) {
    if (bytes <= b.bytes) return OCT_OK;
    drop_graphs(e);
    size_t want = bytes < 256 ? 256 : bytes;
    if (b.bytes && want < b.bytes + b.bytes / 2) want = b.bytes + b.bytes / 2;
    if (b.ptr) EK(cudaFreeAsync(b.ptr, e->stream));
    b.ptr = nullptr;
    b.bytes = 0;
    void* p = nullptr;
    cudaError_t r = cudaMallocFromPoolAsync(&p, want, e->pool, e->stream);
    if (r != cudaSuccess) {
        cudaGetLastError();
        want = bytes;
        r = cudaMallocFromPoolAsync(&p, want, e->pool, e->stream);
    }
    EK(r);
    b.ptr = p;
    b.bytes = want;
    return OCT_OK;
}

int grow_pinned(oct_engine e, size_t bytes) {
    if (bytes <= e->h_stage_bytes) return OCT_OK;
    const size_t want = std::max(bytes, std::max((size_t)256 << 10, e->h_stage_bytes * 2));
    if (e->h_stage) cudaFreeHost(e->h_stage);
    e->h_stage = nullptr;
    e->h_stage_bytes = 0;
    EK(cudaMallocHost(reinterpret_cast<void**>(&e->h_stage), want));
    e->h_stage_bytes = want;
    return OCT_OK;
}

size_t table_offset() { return (sizeof(EngineDyn) + 255) & ~(size_t)255; }

ChunkArgs chunk_args(oct_engine e) {
    const uint64_t cap = std::min<uint64_t>(e->ck_next.bytes / 4, e->ck_pool.bytes / (4ull * kResultChunk));
    return ChunkArgs{e->ck_pool.as<uint32_t>(), e->ck_next.as<uint32_t>(), e->ck_first.as<uint32_t>(),
                     e->ck_ctr.as<uint32_t>(), (uint32_t)std::min<uint64_t>(cap, 0xfffffff0ull)};
}

// Result chunks for `chunks` chunks (grows both arrays; a new address drops the graphs).
int grow_chunks(oct_engine e, uint64_t chunks);

// The launch sequence of the batch in the descriptor (captured or direct).
cudaError_t enqueue_work(oct_engine e) {
    cudaError_t r;
    cudaStream_t s = e->stream;
    EngineDyn* dyn = e->desc.as<EngineDyn>();
    const SearchReq* table = reinterpret_cast<const SearchReq*>(e->desc.as<unsigned char>() + table_offset());
    Summary* sum = e->summary.as<Summary>();
    uint32_t* err = &sum->err;
    SortCtl* ctl = e->sort_ctl.as<SortCtl>();
    // a batch on one cloud: its pointers go to the kernels as parameters
    SearchReq one_req{};
    one_req.cv = e->one_view;
    const SearchReq* one = e->one_cloud ? &one_req : nullptr;
    if ((r = cudaMemsetAsync(sum, 0, sizeof(Summary), s)) != cudaSuccess) return r;
    if ((r = cudaMemsetAsync(ctl, 0, sizeof(SortCtl), s)) != cudaSuccess) return r;
    k_epoch_advance<<<1, 1, 0, s>>>(e->epoch.as<uint32_t>());
    const uint64_t cap_n = e->keys[0].bytes / 8;
    const uint64_t want = (cap_n + kKeyThreads - 1) / kKeyThreads;
    const int kgrid = (int)std::min<uint64_t>(want ? want : 1, (uint64_t)e->sms * 4);
    k_batch_keys<<<kgrid, kKeyThreads, 0, s>>>(dyn, table, e->keys[0].as<uint64_t>(), ctl, e->passes);
    uint32_t* order = nullptr;
    if ((r = launch_sort_dyn(e->device, s, e->keys[0].as<uint64_t>(), e->keys[1].as<uint64_t>(),
                             e->ord[0].as<uint32_t>(), e->ord[1].as<uint32_t>(), &dyn->n_total, cap_n, e->passes,
                             ctl, e->sort_status.as<unsigned long long>(), e->epoch.as<uint32_t>(), err,
                             &order)) != cudaSuccess)
        return r;
    const uint64_t radius_bits = (1ull << kRadiusVariants) - 1;
    const bool any_radius = (e->sig & radius_bits) != 0;
    const bool any_knn = ((e->sig >> kRadiusVariants) & ((1ull << kKnnVariants) - 1)) != 0;
    uint32_t* ctr = e->ctrs.as<uint32_t>();
    unsigned long long* stats = e->stats.as<unsigned long long>();
    const bool fork = any_knn && !e->serial;
    auto knn_groups = [&](cudaStream_t ks) -> cudaError_t {
        cudaError_t r2 = cudaSuccess;
        for (int v = 0; v < kKnnVariants && r2 == cudaSuccess; ++v) {
            if (!((e->sig >> (kRadiusVariants + v)) & 1ull)) continue;
            if (v < 2 && e->knn_group)
                r2 = launch_knn_group_table(e->device, ks, &dyn->groups[kRadiusVariants + v], &dyn->fb[v], one,
                                            32u << v, order, e->bucket, e->knn_idx.as<uint32_t>(),
                                            e->knn_d2.as<double>(), e->knn_counts.as<uint32_t>(), err,
                                            ctr + 2 * kRadiusVariants + 4 * v, e->knn_fb.as<uint32_t>(),
                                            kKnnEstimate, kKnnGroupChunk, e->knn_bps, e->knn_heads.as<double>(),
                                            e->knn_heads.bytes, fp32_on_knn(e->fp32), stats + 2);
            else
                r2 = launch_knn_table(e->device, ks, &dyn->groups[kRadiusVariants + v], one, 0, 32u << v,
                                      order, e->bucket, e->knn_idx.as<uint32_t>(), e->knn_d2.as<double>(),
                                      e->knn_counts.as<uint32_t>(), err, e->knn_bps, kKnnEstimate);
        }
        return r2;
    };
    if (fork) {
        if ((r = cudaEventRecord(e->ev_fork, s)) != cudaSuccess) return r;
        if ((r = cudaStreamWaitEvent(e->side, e->ev_fork, 0)) != cudaSuccess) return r;
        if ((r = knn_groups(e->side)) != cudaSuccess) return r;
        if ((r = cudaEventRecord(e->ev_join, e->side)) != cudaSuccess) return r;
    }
    if (any_radius) {
        unsigned long long* counts = e->counts.as<unsigned long long>();
        unsigned long long* offs = e->offs.as<unsigned long long>();
        unsigned long long* part = e->part.as<unsigned long long>();
        auto scan = [&]() {
            k_escan_reduce<<<kScanBlocks, kScanThreads, 0, s>>>(counts, &dyn->n_radius, part);
            k_escan_top<<<1, kScanThreads, 0, s>>>(part, kScanBlocks, sum);
            k_escan_apply<<<kScanBlocks, kScanThreads, 0, s>>>(counts, &dyn->n_radius, part, offs);
        };
        // one traversal: results into chunk chains, scan, chains compacted into the result array
        const ChunkArgs ck = chunk_args(e);
        if ((r = cudaMemsetAsync(ck.ctr, 0, 4, s)) != cudaSuccess) return r;
        for (int v = 0; v < kRadiusVariants; ++v) {
            if (!((e->sig >> v) & 1ull)) continue;
            const int kernel = v >> 2, algo = (v & 2) ? OCT_NEIGHBORS_PRUNE : OCT_NEIGHBORS;
            if ((r = launch_radius_table(e->device, s, kernel, algo, 2, (v & 1) != 0, &dyn->groups[v], one, 0, order,
                                         counts, nullptr, nullptr, nullptr, 0, ctr + 2 * v, stats, err,
                                         e->radius_bps, &ck)) != cudaSuccess)
                return r;
        }
        scan();
        if ((r = launch_chunk_compact(e->device, s, counts, offs, ck, e->out.as<uint32_t>(), e->out.bytes / 4, 0,
                                      &dyn->n_radius, err)) != cudaSuccess)
            return r;
        const int tb = 128;
        const uint32_t cap_req = (uint32_t)(e->totals.bytes / sizeof(ReqTotal));
        k_req_totals<<<(cap_req + tb - 1) / tb, tb, 0, s>>>(dyn, table, offs, e->totals.as<ReqTotal>());
    }
    if (any_knn && !fork && (r = knn_groups(s)) != cudaSuccess) return r;
    if (fork && (r = cudaStreamWaitEvent(s, e->ev_join, 0)) != cudaSuccess) return r;
    if ((r = cudaMemcpyAsync(e->h_summary, sum, sizeof(Summary), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return r;
    return cudaGetLastError();
}

// Captured graphs kept per engine (a shape is its request variants, sort passes
// and, for a single-cloud batch, the cloud).
constexpr size_t kGraphCache = 1024;

// Launch the current batch: the captured graph of its shape (captured now if
// new) or the direct sequence.
int launch_batch(oct_engine e, bool record_start) {
    DeviceGuardE g(e->device);
    if (e->host_epoch + kEpochStep > kEpochLimit) {  // the look-back epochs wrap: clear the status words
        EK(cudaMemsetAsync(e->sort_status.ptr, 0, e->sort_status.bytes, e->stream));
        EK(cudaMemsetAsync(e->epoch.ptr, 0, 4, e->stream));
        e->host_epoch = 0;
    }
    e->host_epoch += kEpochStep;
    if (record_start) EK(cudaEventRecord(e->ev_t0, e->stream));
    const bool use_graph = !(e->flags & OCT_ENGINE_NO_GRAPH) && e->stream != nullptr;
    if (!use_graph) {
        EK(enqueue_work(e));
    } else {
        const uint64_t key = e->sig;
        cudaGraphExec_t exec = nullptr;
        for (auto& p : e->graphs)
            if (p.sig == key && p.one_cloud == e->one_cloud &&
                (!e->one_cloud || std::memcmp(&p.view, &e->one_view, sizeof(CloudView)) == 0))
                exec = p.exec;
        if (!exec) {
            // keep the cache bounded (the oldest graph goes), but large enough for every shape a
            // serving mix produces: an instantiation now and then takes tens of ms instead of ~0.2
            if (e->graphs.size() >= kGraphCache) {
                cudaGraphExecDestroy(e->graphs.front().exec);
                e->graphs.erase(e->graphs.begin());
            }
            cudaGraph_t graph = nullptr;
            EK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
            const cudaError_t r = enqueue_work(e);
            const cudaError_t r2 = cudaStreamEndCapture(e->stream, &graph);
            if (r != cudaSuccess) {
                if (graph) cudaGraphDestroy(graph);
                return cuda_fail_e(e, r, "capture of the batch sequence");
            }
            EK(r2);
            const cudaError_t r3 = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            EK(r3);
            e->graphs.push_back({key, e->one_cloud, e->one_view, exec});
        }
        EK(cudaGraphLaunch(exec, e->stream));
    }
    EK(cudaEventRecord(e->ev_t1, e->stream));
    if (e->nreq && (e->sig & ((1ull << kRadiusVariants) - 1)))
        EK(cudaMemcpyAsync(e->h_totals, e->totals.ptr, sizeof(ReqTotal) * e->nreq, cudaMemcpyDeviceToHost,
                           e->stream));
    return OCT_OK;
}

int grow_chunks(oct_engine e, uint64_t chunks) {
    if (chunks > 0xfffffff0ull) return fail(e, OCT_ERR_INVALID_ARG, "too many radius results for one batch");
    int st;
    if ((st = grow(e, e->ck_next, 4 * chunks)) != OCT_OK) return st;
    return grow(e, e->ck_pool, 4ull * kResultChunk * chunks);
}

int finish(oct_engine e) {
    DeviceGuardE g(e->device);
    e->in_flight = false;
    for (int attempt = 0; attempt < 4; ++attempt) {
        EK(cudaStreamSynchronize(e->stream));
        const Summary sm = *e->h_summary;
        const uint64_t cap = e->out.bytes / 4;
        const uint32_t grow_bits = (uint32_t)kErrOutputCapacity | (uint32_t)kErrChunkCapacity;
        const uint32_t bits = sm.err & ~grow_bits;
        if (bits & kErrBadInput) return fail(e, OCT_ERR_INVALID_ARG, "device rejected an input");
        if (bits) {
            char buf[128];
            snprintf(buf, sizeof(buf), "a bounded device loop hit its limit (error bits 0x%x)", bits);
            return fail(e, OCT_ERR_DEVICE_LIMIT, buf);
        }
        if (sm.radius_total <= cap && !(sm.err & grow_bits)) {
            e->radius_total = sm.radius_total;
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, e->ev_t0, e->ev_t1) == cudaSuccess) e->last_ms = ms;
            for (size_t i = 0; i < e->places.size(); ++i) {
                const int32_t row = e->place_row[i];
                if (row >= 0 && e->place_type[i] == OCT_REQ_RADIUS) {
                    e->places[i].out_begin = e->h_totals[row].begin;
                    e->places[i].n_results = e->h_totals[row].count;
                }
            }
            e->have_results = true;
            return OCT_OK;
        }
        // the results did not fit: grow the result array (and the chunk pool: every
        // query's last chunk may be partial) to at least twice its size and the exact
        // total, and run the batch again
        const uint64_t want = std::max<uint64_t>(2 * cap, sm.radius_total + sm.radius_total / 8 + 1024);
        int st = grow(e, e->out, 4 * (size_t)want);
        if (st != OCT_OK) return st;
        if ((st = grow_chunks(e, want / kResultChunk + e->n_radius + 1024)) != OCT_OK) return st;
        if ((st = launch_batch(e, true)) != OCT_OK) return st;
    }
    return fail(e, OCT_ERR_CAPACITY, "radius results kept outgrowing the result array");
}

int validate(oct_engine e, const oct_request& r) {
    if (!r.cloud) return fail(e, OCT_ERR_INVALID_ARG, "request without a cloud");
    const Cloud& c = r.cloud->c;
    if (!c.built) return fail(e, OCT_ERR_STATE, "request on a cloud that is not built");
    if (c.device != e->device) return fail(e, OCT_ERR_INVALID_ARG, "cloud on another device than the engine");
    if (r.nq && !r.centers) return fail(e, OCT_ERR_INVALID_ARG, "centers is NULL");
    if (r.type == OCT_REQ_RADIUS) {
        if (r.kernel < OCT_KERNEL_CIRCLE || r.kernel > OCT_KERNEL_CUBE)
            return fail(e, OCT_ERR_INVALID_ARG, "bad kernel");
        if (r.algo != OCT_NEIGHBORS && r.algo != OCT_NEIGHBORS_PRUNE)
            return fail(e, OCT_ERR_INVALID_ARG, "batched radius requests take neighbors or neighborsPrune");
    } else if (r.type == OCT_REQ_KNN) {
        if (r.k < 1 || r.k > 1024) return fail(e, OCT_ERR_INVALID_ARG, "batched kNN takes 1 <= k <= 1024");
    } else {
        return fail(e, OCT_ERR_INVALID_ARG, "bad request type");
    }
    return OCT_OK;
}

int submit(oct_engine e, const oct_request* rq, uint32_t n) {
    int st;
    DeviceGuardE g(e->device);
    if (e->in_flight && (st = finish(e)) != OCT_OK) return st;
    e->have_results = false;
    for (uint32_t i = 0; i < n; ++i)
        if ((st = validate(e, rq[i])) != OCT_OK) return st;
    // variant of every request; non-empty requests in variant order (stable)
    std::vector<int> var(n);
    std::vector<uint32_t> rows;
    rows.reserve(n);
    for (uint32_t i = 0; i < n; ++i) {
        int kv = 0;
        while (rq[i].type == OCT_REQ_KNN && (32u << kv) < rq[i].k) ++kv;
        var[i] = rq[i].type == OCT_REQ_RADIUS ? radius_variant(rq[i].kernel, rq[i].algo, fp32_on_radius(e->fp32))
                                              : kRadiusVariants + kv;
        if (rq[i].nq) rows.push_back(i);
    }
    std::stable_sort(rows.begin(), rows.end(), [&](uint32_t a, uint32_t b) { return var[a] < var[b]; });
    const uint32_t m = (uint32_t)rows.size();
    if (m > (1u << 16)) return fail(e, OCT_ERR_INVALID_ARG, "more than 65536 non-empty requests in one batch");
    // FP32 filter: the leaf-relative copies of the clouds the radius requests read,
    // the centre-relative copies of those the group kNN (k <= 64) reads
    if (e->fp32) {
        for (uint32_t i : rows) {
            Cloud& c = rq[i].cloud->c;
            const bool radius = rq[i].type == OCT_REQ_RADIUS;
            if (radius ? (c.rel_built || !fp32_on_radius(e->fp32))
                       : (c.crel_built || !fp32_on_knn(e->fp32) || !e->knn_group || rq[i].k > 64))
                continue;
            DeviceGuardE gc(c.device);
            if (radius) {
                EK(launch_leaf_rel(c));
                EK(cudaStreamSynchronize(c.stream));
                c.rel_built = true;
            } else {
                EK(launch_center_rel(c));
                EK(cudaStreamSynchronize(c.stream));
                c.crel_built = true;
            }
        }
    }
    // sizes, then capacities (growing drops graphs), then the packed table
    uint64_t n_total = 0, n_radius = 0, knn_slots = 0;
    for (uint32_t i : rows) {
        n_total += rq[i].nq;
        if (rq[i].type == OCT_REQ_RADIUS) n_radius += rq[i].nq;
        else knn_slots += rq[i].nq * rq[i].k;
    }
    if (n_total >= (1ull << 32)) return fail(e, OCT_ERR_INVALID_ARG, "more than 2^32 - 1 centres in one batch");
    const size_t tbl = table_offset();
    const size_t desc_bytes = tbl + (size_t)std::max<uint32_t>(m, 1) * sizeof(SearchReq);
    const uint64_t tiles = (std::max<uint64_t>(n_total, 1) + sort_tile_keys() - 1) / sort_tile_keys();
    const size_t status_before = e->sort_status.bytes;
    if ((st = grow(e, e->desc, desc_bytes)) != OCT_OK) return st;
    for (int b = 0; b < 2; ++b) {
        if ((st = grow(e, e->keys[b], 8 * std::max<uint64_t>(n_total, 1))) != OCT_OK) return st;
        if ((st = grow(e, e->ord[b], 4 * std::max<uint64_t>(n_total, 1))) != OCT_OK) return st;
    }
    // the look-back words cover the key capacity (the sort grid is sized from it)
    const uint64_t cap_tiles = (e->keys[0].bytes / 8 + sort_tile_keys() - 1) / sort_tile_keys();
    if ((st = grow(e, e->sort_status, 256 * 8 * std::max(tiles, cap_tiles))) != OCT_OK) return st;
    if (e->sort_status.bytes != status_before) {
        EK(cudaMemsetAsync(e->sort_status.ptr, 0, e->sort_status.bytes, e->stream));
        EK(cudaMemsetAsync(e->epoch.ptr, 0, 4, e->stream));
        e->host_epoch = 0;
    }
    if ((st = grow(e, e->counts, 8 * std::max<uint64_t>(n_radius, 1))) != OCT_OK) return st;
    if ((st = grow(e, e->offs, 8 * (n_radius + 1))) != OCT_OK) return st;
    if ((st = grow(e, e->knn_idx, 4 * std::max<uint64_t>(knn_slots, 1))) != OCT_OK) return st;
    if ((st = grow(e, e->knn_d2, 8 * std::max<uint64_t>(knn_slots, 1))) != OCT_OK) return st;
    if ((st = grow(e, e->knn_counts, 4 * std::max<uint64_t>(n_total, 1))) != OCT_OK) return st;
    if (knn_slots && e->knn_group) {
        if ((st = grow(e, e->knn_fb, 4 * n_total)) != OCT_OK) return st;
        // heads: one per kKnnHeadStride groups of every request (each request's groups round up)
        const uint64_t groups = n_total / kKnnGroupQueries + m;
        if ((st = grow(e, e->knn_heads, 8 * (groups / kKnnHeadStride + 2))) != OCT_OK) return st;
    }
    if ((st = grow(e, e->totals, sizeof(ReqTotal) * std::max<uint32_t>(m, 1))) != OCT_OK) return st;
    if (n_radius) {  // one-pass radius: a first chunk per query, a pool of at least 3 chunks per query
        if ((st = grow(e, e->ck_first, 4 * n_radius)) != OCT_OK) return st;
        if ((st = grow(e, e->ck_ctr, 256)) != OCT_OK) return st;
        const uint64_t have = chunk_args(e).cap;
        const uint64_t want = std::max<uint64_t>(3 * n_radius + 1024, e->out.bytes / (4ull * kResultChunk) + n_radius);
        if (have < want && (st = grow_chunks(e, want)) != OCT_OK) return st;
    }
    if (e->out.bytes == 0 && (st = grow(e, e->out, 4 * std::max<uint64_t>(64 * n_radius, 1u << 20))) != OCT_OK)
        return st;
    if (m > e->h_totals_cap) {
        if (e->h_totals) cudaFreeHost(e->h_totals);
        e->h_totals = nullptr;
        e->h_totals_cap = 0;
        const size_t want = std::max<size_t>(m, 1024);
        EK(cudaMallocHost(reinterpret_cast<void**>(&e->h_totals), sizeof(ReqTotal) * want));
        e->h_totals_cap = want;
    }
    if ((st = grow_pinned(e, desc_bytes)) != OCT_OK) return st;
    // the pinned staging may still feed the previous batch's copy
    EK(cudaStreamSynchronize(e->stream));
    std::memset(e->h_stage, 0, tbl);
    EngineDyn* dyn = reinterpret_cast<EngineDyn*>(e->h_stage);
    SearchReq* table = reinterpret_cast<SearchReq*>(e->h_stage + tbl);
    const SearchReq* d_table = reinterpret_cast<const SearchReq*>(e->desc.as<unsigned char>() + tbl);
    e->places.assign(n, oct_request_place{0, 0, 0, 0});
    e->place_row.assign(n, -1);
    e->place_type.assign(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
        e->place_type[i] = rq[i].type;
        e->places[i].nq = rq[i].nq;
    }
    std::unordered_map<const Cloud*, uint32_t> cloud_ids;
    uint64_t sig = 0, pos = 0, slot = 0;
    for (uint32_t t = 0; t < m;) {
        const int v = var[rows[t]];
        DynGroup& gr = dyn->groups[v];
        gr.reqs = d_table + t;
        gr.q_begin = pos;
        gr.kmax = 0;
        // packets: 32 queries (radius), kKnnGroupQueries (group kNN); the per-query kNN kernel ignores them
        const bool group_knn = e->knn_group && v >= kRadiusVariants && v < kRadiusVariants + 2;
        const uint64_t per = group_knn ? kKnnGroupQueries : 32;
        uint32_t t0 = t;
        for (; t < m && var[rows[t]] == v; ++t) {
            const uint32_t i = rows[t];
            const oct_request& r = rq[i];
            const Cloud& c = r.cloud->c;
            auto it = cloud_ids.find(&c);
            const uint32_t cid = it != cloud_ids.end() ? it->second : (uint32_t)cloud_ids.size();
            if (it == cloud_ids.end()) cloud_ids.emplace(&c, cid);
            SearchReq s{};
            s.cv = cloud_view(c);
            s.centers = r.centers;
            s.radii = r.type == OCT_REQ_RADIUS ? r.radii : nullptr;
            s.radius = r.radius;
            s.q_begin = pos;
            s.q_end = pos + r.nq;
            s.packet_begin = gr.packets;
            s.cloud_id = cid;
            if (r.type == OCT_REQ_KNN) {
                s.k = r.k;
                s.out_begin = slot;
                e->places[i].out_begin = slot;
                slot += r.nq * r.k;
                gr.kmax = std::max(gr.kmax, r.k);
            }
            table[t] = s;
            e->places[i].q_begin = pos;
            e->place_row[i] = (int32_t)t;
            gr.packets += (r.nq + per - 1) / per;
            pos += r.nq;
        }
        gr.nreq = t - t0;
        gr.nq = pos - gr.q_begin;
        if (group_knn) {  // the fallback group: the same requests, its count starts at 0
            DynGroup& fb = dyn->fb[v - kRadiusVariants];
            fb.reqs = gr.reqs;
            fb.nreq = gr.nreq;
            fb.kmax = gr.kmax;
            fb.q_begin = gr.q_begin;
        }
        sig |= 1ull << v;
    }
    dyn->n_total = n_total;
    dyn->n_radius = n_radius;
    dyn->nreq = m;
    // one cloud: the kernels take its pointers as parameters (the graph is kept per cloud view)
    e->one_cloud = cloud_ids.size() == 1;
    if (e->one_cloud) e->one_view = cloud_view(*cloud_ids.begin()->first);
    int req_bits = 0;
    while (m > 1 && (1u << req_bits) < m) ++req_bits;
    e->passes = 3 + (req_bits + 7) / 8;
    e->sig = sig | ((uint64_t)e->passes << 32) | ((uint64_t)e->fp32 << 40);
    e->n_total = n_total;
    e->n_radius = n_radius;
    e->knn_slots = knn_slots;
    e->nreq = m;
    e->desc_bytes = desc_bytes;
    EK(cudaEventRecord(e->ev_t0, e->stream));  // the batch's device time starts with its descriptor copy
    EK(cudaMemcpyAsync(e->desc.ptr, e->h_stage, tbl + (size_t)m * sizeof(SearchReq), cudaMemcpyHostToDevice,
                       e->stream));
    if (m == 0) {  // nothing to search
        e->h_summary->radius_total = 0;
        e->h_summary->err = 0;
        e->radius_total = 0;
        e->have_results = true;
        return OCT_OK;
    }
    if ((st = launch_batch(e, false)) != OCT_OK) return st;
    e->in_flight = true;
    return OCT_OK;
}

void write_places(oct_engine e, oct_request_place* places) {
    if (!places) return;
    for (size_t i = 0; i < e->places.size(); ++i) places[i] = e->places[i];
}

}  // namespace

extern "C" {

int oct_engine_create(const oct_engine_params* p, oct_engine* out) {
    if (!p || !out) return OCT_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return OCT_ERR_NO_DEVICE;
    }
    if (p->device < 0 || p->device >= ndev) return OCT_ERR_INVALID_ARG;
    oct_engine e = new (std::nothrow) oct_engine_s();
    if (!e) return OCT_ERR_OUT_OF_MEMORY;
    e->device = p->device;
    e->flags = p->flags;
    DeviceGuardE g(e->device);
    e->sms = sm_count_e(e->device);
    cudaError_t r = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (r == cudaSuccess) {
        e->own_stream = true;
        r = cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking);
    }
    if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming);
    if (r == cudaSuccess) r = cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming);
    if (r == cudaSuccess) r = cudaEventCreate(&e->ev_t0);
    if (r == cudaSuccess) r = cudaEventCreate(&e->ev_t1);
    if (r == cudaSuccess) r = prepare_sort_dyn();
    if (r == cudaSuccess) r = prepare_knn_dyn();
    // every kernel loaded now, not at its first launch in the middle of a stream of batches
    if (r == cudaSuccess && preload_kernels(e->device) != OCT_OK) r = cudaErrorInitializationError;
    if (r == cudaSuccess) r = e->sort_ctl.reserve(sizeof(SortCtl));
    if (r == cudaSuccess) r = e->epoch.reserve(256);
    if (r == cudaSuccess) r = e->ctrs.reserve(4 * (2 * kRadiusVariants + 4 * 2));  // + group kNN (3 of 4 per variant)
    if (r == cudaSuccess) r = e->stats.reserve(64);
    if (r == cudaSuccess) r = e->summary.reserve(256);
    if (r == cudaSuccess) r = e->part.reserve(8 * (kScanBlocks + 1));
    if (r == cudaSuccess) r = cudaMemsetAsync(e->epoch.ptr, 0, 256, e->stream);
    if (r == cudaSuccess) r = cudaMemsetAsync(e->stats.ptr, 0, 64, e->stream);
    if (r == cudaSuccess) r = cudaMallocHost(reinterpret_cast<void**>(&e->h_summary), sizeof(Summary));
    if (r == cudaSuccess) {  // the pool of the growable arrays: keeps what it frees, for the next growth
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = e->device;
        r = cudaMemPoolCreate(&e->pool, &props);
        uint64_t keep = UINT64_MAX;
        if (r == cudaSuccess) r = cudaMemPoolSetAttribute(e->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (r == cudaSuccess && p->reserve_results && grow(e, e->out, 4 * p->reserve_results) != OCT_OK)
        r = cudaErrorMemoryAllocation;
    if (r == cudaSuccess && p->reserve_queries) {  // a batch of this many centres grows nothing of these
        const uint64_t q = p->reserve_queries;
        DevBuf* per_q8[] = {&e->keys[0], &e->keys[1], &e->counts, &e->offs};
        for (DevBuf* b : per_q8)
            if (r == cudaSuccess && grow(e, *b, 8 * (q + 1)) != OCT_OK) r = cudaErrorMemoryAllocation;
        DevBuf* per_q4[] = {&e->ord[0], &e->ord[1], &e->knn_counts, &e->knn_fb, &e->ck_first};
        for (DevBuf* b : per_q4)
            if (r == cudaSuccess && grow(e, *b, 4 * (q + 1)) != OCT_OK) r = cudaErrorMemoryAllocation;
        // kNN results of up to 256 neighbours per centre, the request table of 1024 requests, the sort's
        // look-back words, the group kNN's heads and the one-pass radius search's chunk pool
        const uint64_t tiles = (q + sort_tile_keys() - 1) / sort_tile_keys();
        const size_t want[][2] = {{0, 4 * q * 256}, {1, 8 * q * 256}, {2, sizeof(ReqTotal) * 1024},
                                  {3, table_offset() + 1024 * sizeof(SearchReq)}, {4, 256 * 8 * tiles},
                                  {5, 8 * (q / kKnnGroupQueries / kKnnHeadStride + 1026)}, {6, 256}};
        DevBuf* bufs[] = {&e->knn_idx, &e->knn_d2, &e->totals, &e->desc, &e->sort_status, &e->knn_heads, &e->ck_ctr};
        for (const auto& w : want)
            if (r == cudaSuccess && grow(e, *bufs[w[0]], w[1]) != OCT_OK) r = cudaErrorMemoryAllocation;
        if (r == cudaSuccess) r = cudaMemsetAsync(e->sort_status.ptr, 0, e->sort_status.bytes, e->stream);
        const uint64_t chunks = std::max<uint64_t>(3 * q + 1024, e->out.bytes / (4ull * kResultChunk) + q);
        if (r == cudaSuccess && grow_chunks(e, chunks) != OCT_OK) r = cudaErrorMemoryAllocation;
        if (r == cudaSuccess && grow_pinned(e, table_offset() + 1024 * sizeof(SearchReq)) != OCT_OK)
            r = cudaErrorMemoryAllocation;
        if (r == cudaSuccess) {
            r = cudaMallocHost(reinterpret_cast<void**>(&e->h_totals), sizeof(ReqTotal) * 1024);
            if (r == cudaSuccess) e->h_totals_cap = 1024;
        }
    }
    if (r == cudaSuccess) r = cudaStreamSynchronize(e->stream);
    if (r != cudaSuccess) {
        cudaGetLastError();
        oct_engine_destroy(e);
        return r == cudaErrorMemoryAllocation ? OCT_ERR_OUT_OF_MEMORY : OCT_ERR_CUDA;
    }
    e->h_summary->radius_total = 0;
    e->h_summary->err = 0;
    *out = e;
    return OCT_OK;
}

int oct_engine_destroy(oct_engine e) {
    if (!e) return OCT_ERR_INVALID_ARG;
    {
        DeviceGuardE g(e->device);
        if (e->stream) cudaStreamSynchronize(e->stream);
        drop_graphs(e);
        DevBuf* fixed[] = {&e->sort_ctl, &e->epoch, &e->part, &e->ctrs, &e->stats, &e->summary};
        for (DevBuf* b : fixed) b->release();
        DevBuf* pooled[] = {&e->desc, &e->keys[0], &e->keys[1], &e->ord[0], &e->ord[1], &e->sort_status,
                            &e->counts, &e->offs, &e->out, &e->knn_idx, &e->knn_d2, &e->knn_counts, &e->totals,
                            &e->ck_pool, &e->ck_next, &e->ck_first, &e->ck_ctr, &e->knn_fb, &e->knn_heads,
                            &e->hash_out};
        for (DevBuf* b : pooled) {
            if (b->ptr && e->stream) cudaFreeAsync(b->ptr, e->stream);
            b->ptr = nullptr;
            b->bytes = 0;
        }
        if (e->stream) cudaStreamSynchronize(e->stream);
        if (e->pool) cudaMemPoolDestroy(e->pool);
        if (e->h_stage) cudaFreeHost(e->h_stage);
        if (e->h_summary) cudaFreeHost(e->h_summary);
        if (e->h_totals) cudaFreeHost(e->h_totals);
        if (e->ev_fork) cudaEventDestroy(e->ev_fork);
        if (e->ev_join) cudaEventDestroy(e->ev_join);
        if (e->ev_t0) cudaEventDestroy(e->ev_t0);
        if (e->ev_t1) cudaEventDestroy(e->ev_t1);
        if (e->side) cudaStreamDestroy(e->side);
        if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    }
    delete e;
    return OCT_OK;
}

int oct_engine_set_stream(oct_engine e, void* stream) {
    if (!e) return OCT_ERR_INVALID_ARG;
    DeviceGuardE g(e->device);
    if (e->in_flight) {
        const int st = finish(e);
        if (st != OCT_OK) return st;
    }
    EK(cudaStreamSynchronize(e->stream));
    if (e->own_stream) cudaStreamDestroy(e->stream);
    e->own_stream = false;
    e->stream = static_cast<cudaStream_t>(stream);
    drop_graphs(e);
    return OCT_OK;
}

int oct_engine_last_error(oct_engine e, char* buf, size_t len) {
    if (!e || !buf || len == 0) return OCT_ERR_INVALID_ARG;
    const size_t k = std::min(len - 1, e->last_error.size());
    memcpy(buf, e->last_error.data(), k);
    buf[k] = '\0';
    return OCT_OK;
}

int oct_engine_set_config(oct_engine e, const oct_search_config* cfg) {
    if (!e || !cfg) return OCT_ERR_INVALID_ARG;
    if (cfg->knn_bucket < 0 || cfg->reserved[0] < 0 || cfg->reserved[0] > 16 || cfg->reserved[1] < 0 ||
        cfg->reserved[1] > 16 || cfg->reserved[2] < 0 || cfg->reserved[2] > 1 || cfg->fp32_filter < 0 ||
        cfg->fp32_filter > OCT_FP32_KNN)
        return fail(e, OCT_ERR_INVALID_ARG, "bad engine configuration");
    if (e->in_flight) {
        const int st = finish(e);
        if (st != OCT_OK) return st;
    }
    const int fp32 = cfg->fp32_filter;
    const uint32_t bucket = (uint32_t)cfg->knn_bucket;
    const int knn_group = cfg->knn_packet ? 1 : 0;
    if (fp32 != e->fp32 || bucket != e->bucket || cfg->reserved[0] != e->radius_bps ||
        cfg->reserved[1] != e->knn_bps || cfg->reserved[2] != e->serial || knn_group != e->knn_group)
        drop_graphs(e);
    e->fp32 = fp32;
    e->bucket = bucket;
    e->radius_bps = cfg->reserved[0];
    e->knn_bps = cfg->reserved[1];
    e->serial = cfg->reserved[2];
    e->knn_group = knn_group;
    return OCT_OK;
}

int oct_engine_get_config(oct_engine e, oct_search_config* cfg) {
    if (!e || !cfg) return OCT_ERR_INVALID_ARG;
    memset(cfg, 0, sizeof(*cfg));
    cfg->packet = 1;
    cfg->fp32_filter = e->fp32;
    cfg->radius_lanes = 32;
    cfg->knn_packet = e->knn_group;
    cfg->knn_bucket = (int32_t)e->bucket;
    cfg->reserved[0] = e->radius_bps;
    cfg->reserved[1] = e->knn_bps;
    cfg->reserved[2] = e->serial;
    return OCT_OK;
}

int oct_engine_submit(oct_engine e, const oct_request* rq, uint32_t n, oct_request_place* places) {
    if (!e || (n && !rq)) return OCT_ERR_INVALID_ARG;
    const int st = submit(e, rq, n);
    if (st == OCT_OK) write_places(e, places);
    return st;
}

int oct_engine_wait(oct_engine e, oct_request_place* places, uint64_t* radius_total) {
    if (!e) return OCT_ERR_INVALID_ARG;
    if (e->in_flight) {
        const int st = finish(e);
        if (st != OCT_OK) return st;
    }
    if (!e->have_results) return fail(e, OCT_ERR_STATE, "no batch submitted");
    write_places(e, places);
    if (radius_total) *radius_total = e->radius_total;
    return OCT_OK;
}

int oct_engine_run(oct_engine e, const oct_request* rq, uint32_t n, oct_request_place* places,
                   uint64_t* radius_total) {
    int st = oct_engine_submit(e, rq, n, nullptr);
    if (st != OCT_OK) return st;
    return oct_engine_wait(e, places, radius_total);
}

int oct_engine_outputs(oct_engine e, uint64_t** offsets, uint32_t** indices, uint32_t** knn_idx, double** knn_d2,
                       uint32_t** knn_counts) {
    if (!e) return OCT_ERR_INVALID_ARG;
    if (e->in_flight || !e->have_results) return fail(e, OCT_ERR_STATE, "no completed batch");
    if (offsets) *offsets = e->offs.as<uint64_t>();
    if (indices) *indices = e->out.as<uint32_t>();
    if (knn_idx) *knn_idx = e->knn_idx.as<uint32_t>();
    if (knn_d2) *knn_d2 = e->knn_d2.as<double>();
    if (knn_counts) *knn_counts = e->knn_counts.as<uint32_t>();
    return OCT_OK;
}

int oct_engine_copy_radius(oct_engine e, const oct_request_place* pl, uint64_t* offsets, uint32_t* idx,
                           uint64_t idx_capacity, uint32_t flags) {
    if (!e || !pl) return OCT_ERR_INVALID_ARG;
    if (e->in_flight || !e->have_results) return fail(e, OCT_ERR_STATE, "no completed batch");
    DeviceGuardE g(e->device);
    const bool dev = (flags & OCT_MEM_DEVICE) != 0;
    const uint64_t nq = pl->nq;
    if (offsets) {
        if (nq == 0) {
            if (dev) EK(cudaMemsetAsync(offsets, 0, 8, e->stream));
            else offsets[0] = 0;
        } else if (pl->q_begin + nq > e->n_radius) {
            return fail(e, OCT_ERR_INVALID_ARG, "place is not a radius request of the last batch");
        } else if (dev) {
            k_rebase<<<(unsigned)((nq + 1 + 255) / 256), 256, 0, e->stream>>>(
                e->offs.as<unsigned long long>() + pl->q_begin, nq + 1, reinterpret_cast<unsigned long long*>(offsets));
            EK(cudaGetLastError());
        } else {
            EK(cudaMemcpyAsync(offsets, e->offs.as<uint64_t>() + pl->q_begin, 8 * (nq + 1), cudaMemcpyDeviceToHost,
                               e->stream));
        }
    }
    const bool fits = idx_capacity >= pl->n_results;
    if (idx && fits && pl->n_results)
        EK(cudaMemcpyAsync(idx, e->out.as<uint32_t>() + pl->out_begin, 4 * pl->n_results,
                           dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, e->stream));
    EK(cudaStreamSynchronize(e->stream));
    if (offsets && !dev && nq) {
        const uint64_t b = offsets[0];
        if (b != 0)  // the batch's first radius request starts at 0 already
            for (uint64_t i = 0; i <= nq; ++i) offsets[i] -= b;
    }
    if (idx && !fits) return fail(e, OCT_ERR_CAPACITY, "idx_capacity smaller than the request's results");
    return OCT_OK;
}

int oct_engine_copy_radius_hash(oct_engine e, const oct_request_place* pl, uint64_t* counts, uint64_t* hashes,
                                uint32_t flags) {
    if (!e || !pl) return OCT_ERR_INVALID_ARG;
    if (e->in_flight || !e->have_results) return fail(e, OCT_ERR_STATE, "no completed batch");
    const uint64_t nq = pl->nq;
    if (nq == 0) return OCT_OK;
    if (!counts || !hashes) return fail(e, OCT_ERR_INVALID_ARG, "counts or hashes is NULL");
    if (pl->q_begin + nq > e->n_radius)
        return fail(e, OCT_ERR_INVALID_ARG, "place is not a radius request of the last batch");
    DeviceGuardE g(e->device);
    const bool dev = (flags & OCT_MEM_DEVICE) != 0;
    unsigned long long* dc = reinterpret_cast<unsigned long long*>(counts);
    unsigned long long* dh = reinterpret_cast<unsigned long long*>(hashes);
    if (!dev) {
        int st;
        if ((st = grow(e, e->hash_out, 16 * nq)) != OCT_OK) return st;
        dc = e->hash_out.as<unsigned long long>();
        dh = dc + nq;
    }
    const uint64_t want = (nq + 7) / 8;
    const uint64_t cap = (uint64_t)e->sms * 8;
    k_csr_hash<<<(unsigned)(want < cap ? want : cap), 256, 0, e->stream>>>(
        e->offs.as<unsigned long long>() + pl->q_begin, e->out.as<uint32_t>(), nq, dc, dh);
    EK(cudaGetLastError());
    if (!dev) {
        EK(cudaMemcpyAsync(counts, dc, 8 * nq, cudaMemcpyDeviceToHost, e->stream));
        EK(cudaMemcpyAsync(hashes, dh, 8 * nq, cudaMemcpyDeviceToHost, e->stream));
    }
    EK(cudaStreamSynchronize(e->stream));
    return OCT_OK;
}

int oct_engine_copy_knn(oct_engine e, const oct_request_place* pl, uint32_t k, uint32_t* idx, double* d2,
                        uint32_t* counts, uint32_t flags) {
    if (!e || !pl) return OCT_ERR_INVALID_ARG;
    if (e->in_flight || !e->have_results) return fail(e, OCT_ERR_STATE, "no completed batch");
    DeviceGuardE g(e->device);
    const bool dev = (flags & OCT_MEM_DEVICE) != 0;
    const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const uint64_t slots = pl->nq * k;
    if (pl->nq && (pl->q_begin < e->n_radius || pl->out_begin + slots > e->knn_slots))
        return fail(e, OCT_ERR_INVALID_ARG, "place is not a kNN request of the last batch with this k");
    if (idx && slots) EK(cudaMemcpyAsync(idx, e->knn_idx.as<uint32_t>() + pl->out_begin, 4 * slots, kind, e->stream));
    if (d2 && slots) EK(cudaMemcpyAsync(d2, e->knn_d2.as<double>() + pl->out_begin, 8 * slots, kind, e->stream));
    if (counts && pl->nq)
        EK(cudaMemcpyAsync(counts, e->knn_counts.as<uint32_t>() + pl->q_begin, 4 * pl->nq, kind, e->stream));
    EK(cudaStreamSynchronize(e->stream));
    return OCT_OK;
}

int oct_engine_last_ms(oct_engine e, float* ms) {
    if (!e || !ms) return OCT_ERR_INVALID_ARG;
    *ms = e->last_ms;
    return OCT_OK;
}

int oct_engine_ready(oct_engine e, int* ready) {
    if (!e || !ready) return OCT_ERR_INVALID_ARG;
    if (!e->in_flight) {
        *ready = 1;
        return OCT_OK;
    }
    DeviceGuardE g(e->device);
    const cudaError_t r = cudaStreamQuery(e->stream);
    if (r == cudaErrorNotReady) {
        *ready = 0;
        return OCT_OK;
    }
    EK(r);
    *ready = 1;
    return OCT_OK;
}

int oct_engine_memory(oct_engine e, uint64_t* bytes) {
    if (!e || !bytes) return OCT_ERR_INVALID_ARG;
    const DevBuf* bufs[] = {&e->desc, &e->keys[0], &e->keys[1], &e->ord[0], &e->ord[1], &e->sort_ctl,
                            &e->sort_status, &e->epoch, &e->counts, &e->offs, &e->part, &e->out, &e->knn_idx,
                            &e->knn_d2, &e->knn_counts, &e->ctrs, &e->stats, &e->summary, &e->totals,
                            &e->ck_pool, &e->ck_next, &e->ck_first, &e->ck_ctr, &e->knn_fb,
                            &e->knn_heads, &e->hash_out};
    uint64_t s = 0;
    for (const DevBuf* b : bufs) s += b->bytes;
    *bytes = s;
    return OCT_OK;
}

int oct_engine_autotune(oct_engine e, const oct_request* rq, uint32_t n, oct_search_config* chosen) {
    if (!e || (n && !rq)) return OCT_ERR_INVALID_ARG;
    int st;
    std::vector<oct_request> radius, knn;
    for (uint32_t i = 0; i < n; ++i) (rq[i].type == OCT_REQ_RADIUS ? radius : knn).push_back(rq[i]);
    // time one configuration on one kind of request: a warm run (captures the
    // graph), then the best of two timed runs
    auto time_cfg = [&](const std::vector<oct_request>& set, float* best) -> int {
        *best = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            int s2 = oct_engine_run(e, set.data(), (uint32_t)set.size(), nullptr, nullptr);
            if (s2 != OCT_OK) return s2;
            if (rep > 0) *best = std::min(*best, e->last_ms);
        }
        return OCT_OK;
    };
    oct_search_config cfg;
    oct_engine_get_config(e, &cfg);
    // the radius filter and the kNN filter are chosen separately (each on its own kind of request)
    bool radius_f32 = fp32_on_radius(cfg.fp32_filter), knn_f32 = fp32_on_knn(cfg.fp32_filter);
    auto combined = [](bool r, bool k) { return r ? (k ? OCT_FP32_ALL : OCT_FP32_RADIUS) : (k ? OCT_FP32_KNN : 0); };
    if (!radius.empty()) {
        const int fp32s[2] = {0, OCT_FP32_RADIUS};
        const int bps[3] = {4, 8, 12};
        float best = 1e30f;
        oct_search_config pick = cfg;
        for (int f : fp32s)
            for (int b : bps) {
                oct_search_config c2 = cfg;
                c2.fp32_filter = f;
                c2.reserved[0] = b;
                if ((st = oct_engine_set_config(e, &c2)) != OCT_OK) return st;
                float t;
                if ((st = time_cfg(radius, &t)) != OCT_OK) return st;
                if (t < best) {
                    best = t;
                    pick = c2;
                }
            }
        radius_f32 = fp32_on_radius(pick.fp32_filter);
        cfg.fp32_filter = combined(radius_f32, knn_f32);
        cfg.reserved[0] = pick.reserved[0];
    }
    if (!knn.empty()) {
        // groups of queries per warp (blocks per SM follow from its shared memory), then one warp per query
        // (the group kernel with and without its FP32 filter)
        struct KnnCfg {
            int group, bucket, bps, f32;
        };
        const KnnCfg cands[12] = {{1, 128, 0, 0},  {1, 256, 0, 0}, {1, 128, 0, 1},  {1, 256, 0, 1},
                                  {0, 0, 8, 0},    {0, 0, 16, 0},  {0, 64, 8, 0},   {0, 64, 16, 0},
                                  {0, 128, 8, 0},  {0, 128, 16, 0}, {0, 256, 8, 0}, {0, 256, 16, 0}};
        float best = 1e30f;
        oct_search_config pick = cfg;
        for (const KnnCfg& kc : cands) {
            oct_search_config c2 = cfg;
            c2.fp32_filter = combined(radius_f32, kc.f32 != 0);
            c2.knn_packet = kc.group;
            c2.knn_bucket = kc.bucket;
            c2.reserved[1] = kc.bps;
            if ((st = oct_engine_set_config(e, &c2)) != OCT_OK) return st;
            float t;
            if ((st = time_cfg(knn, &t)) != OCT_OK) return st;
            if (t < best) {
                best = t;
                pick = c2;
            }
        }
        knn_f32 = fp32_on_knn(pick.fp32_filter);
        cfg.fp32_filter = combined(radius_f32, knn_f32);
        cfg.knn_packet = pick.knn_packet;
        cfg.knn_bucket = pick.knn_bucket;
        cfg.reserved[1] = pick.reserved[1];
    }
    if (!radius.empty() && !knn.empty()) {  // kNN beside the radius search, or after it
        std::vector<oct_request> all(rq, rq + n);
        float best = 1e30f;
        int pick = 0;
        for (int ser = 0; ser < 2; ++ser) {
            oct_search_config c2 = cfg;
            c2.reserved[2] = ser;
            if ((st = oct_engine_set_config(e, &c2)) != OCT_OK) return st;
            float t;
            if ((st = time_cfg(all, &t)) != OCT_OK) return st;
            if (t < best) {
                best = t;
                pick = ser;
            }
        }
        cfg.reserved[2] = pick;
    }
    if ((st = oct_engine_set_config(e, &cfg)) != OCT_OK) return st;
    if (chosen) *chosen = cfg;
    return OCT_OK;
}

}  // extern "C"
