// Host-side state of one device-resident cloud (the object behind oct_cloud)
// and the launchers each .cu file provides.  Internal to the library.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/octree_b200.h"
#include "oct_common.cuh"

namespace octb {

// A grow-only device allocation.  Bound to a memory pool and a stream (a
// cloud's arrays), its storage comes from the pool in that stream's order
// (cudaMallocFromPoolAsync / cudaFreeAsync): building or destroying a cloud
// then waits for nothing but its own stream, where cudaMalloc / cudaFree would
// wait for all work on the device (every other cloud's and engine's).
// Unbound, it uses cudaMalloc / cudaFree.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaMemPool_t pool = nullptr;
    const cudaStream_t* stream = nullptr;  // the owner's current stream (followed when the owner switches it)
    void bind(cudaMemPool_t p, const cudaStream_t* s) {
        pool = p;
        stream = s;
    }
    cudaError_t reserve(size_t want) {
        if (want <= bytes) return cudaSuccess;
        release();
        size_t b = want < 256 ? 256 : want;
        cudaError_t e = pool ? cudaMallocFromPoolAsync(&ptr, b, pool, *stream) : cudaMalloc(&ptr, b);
        if (e == cudaSuccess) bytes = b;
        else ptr = nullptr;
        return e;
    }
    void release() {
        if (ptr) {
            if (pool) cudaFreeAsync(ptr, *stream);
            else cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
};

// The memory pool of every cloud's arrays on a device (created on first use,
// kept for the process; it holds up to 8 GB of freed storage for reuse).
cudaMemPool_t cloud_pool(int device);
// Pinned host blocks of kPinnedBlock bytes, reused across clouds (cudaFreeHost can wait for the device).
constexpr size_t kPinnedBlock = 4096;
void* pinned_block_get();
void pinned_block_put(void* p);

// Device-side record of the sort (one per cloud): the 8 digit histograms of
// the keys, their exclusive scans, which passes are skipped (all keys share
// the digit) and one tile counter per pass.
struct SortCtl {
    unsigned long long offs[8][256];
    uint32_t hist[8][256];
    uint32_t skip[8];
    uint32_t tile_ctr[8];
    uint32_t bbox_ctr;
    uint32_t pad;
};

// Octree build bookkeeping written by the device.
struct BuildCtl {
    uint32_t level_start[kMaxDepth + 3];  // first node index of each level
    uint32_t level_internal[kMaxDepth + 2];
    uint32_t n_total;
    uint32_t n_internal;
    uint32_t max_depth_seen;
    uint32_t need_nodes;                  // nodes the tree needs (valid when kErrNodeCapacity)
    uint32_t barrier_count;
    uint32_t barrier_gen;
};

// Device pointers of one built cloud, as the search kernels read them.
struct CloudView {
    const double* xs;
    const double* ys;
    const double* zs;
    const float4* rel;          // FP32 leaf-relative points (packet FP32 path), may be null
    const float4* crel;         // FP32 points relative to the box centre (group kNN FP32 path), may be null
    const uint32_t* offsets;
    const uint2* ranges;
    const double* centers;
    const LevelGeom* geom;      // per-level radii
    const BoxD* box;            // the cloud's Box (anchor frame of its keys)
    int32_t encoder;            // OCT_ENC_MORTON_3D or OCT_ENC_HILBERT_3D
    uint32_t pad;
};

// One request of a search launch (device copy).  A launch covers a table of
// requests; every query of the launch has a global position q in
// [q_begin, q_end) of its request, and outputs are indexed by q.
struct SearchReq {
    CloudView cv;
    const double* centers;      // the request's nq x 3 centres
    const double* radii;        // per-query radii (radius requests) or null
    double radius;              // radius when radii is null
    uint64_t q_begin, q_end;    // global query positions of this request
    uint64_t packet_begin;      // first packet (32 queries) of the request in the launch
    uint64_t out_begin;         // kNN: first output slot (previous requests' nq * k)
    uint32_t k;                 // kNN k
    uint32_t cloud_id;          // distinct per cloud within the table (radii reload key)
    uint32_t approx_cut;        // neighborsStruct: 0, or neighborsApprox's precisionLevel + 1
    uint32_t approx_upper;      // neighborsApprox: 1 adds the ranges of the cut octants
};

// Launch sizes of one kernel group of a batch, in device memory.  The host
// writes them before the batch runs, so one launch configuration (and one
// captured graph) serves batches of any size.
struct DynGroup {
    const SearchReq* reqs;      // the group's requests (device), positions ascending
    uint32_t nreq;
    uint32_t kmax;              // kNN: largest k of the group
    uint64_t packets;           // radius: 32-query packets of the group
    uint64_t q_begin;           // first query position of the group
    uint64_t nq;                // queries of the group
};

// Register kNN: provisional k-th distance = this factor x the radius that holds k
// points at the density of the query's first cell (exact either way).
constexpr double kKnnEstimate = 1.2;
// Group kNN: consecutive query groups a warp takes at a time (the later ones start
// from the previous group's k-th distances).
constexpr uint32_t kKnnGroupChunk = 4;
// group kNN heads: every kKnnHeadStride-th group is searched first, from the
// density estimate; the others start from a neighbouring group's k-th distance
constexpr uint32_t kKnnHeadStride = 16;
// Queries per warp of the group kNN (4 or 8).  4: half the shared memory per
// warp, so 28 warps per SM instead of 16, for ~1.6x the node visits per query;
// ~20 % faster on the 10M-point tile (k = 50).
constexpr uint32_t kKnnGroupQueries = 4;

struct Cloud {
    oct_params params{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint64_t n = 0;
    bool sorted = false;
    bool built = false;
    int radius_group = 8;
    std::string last_error;

    // points
    DevBuf xyz_in;          // AoS input (n x 3 f64), as uploaded
    DevBuf xs, ys, zs;      // SFC-sorted coordinates, SoA f64
    DevBuf keys, keys_alt;  // u64 keys (sorted result lives in `keys`)
    DevBuf perm, perm_alt;  // u32 input position of each sorted point
    DevBuf keys_hi, keys_hi_alt;  // u32 upper key halves (the split sort)
    DevBuf run_pv, run_pv_alt;    // u64 lower key half << 32 | input position (the split sort)
    DevBuf run_ctl, run_list;     // the split sort's run bookkeeping
    DevBuf run_long;              // its runs longer than 4096 points (LongRun entries)
    int split_sel = 0;            // which keys_hi / run_pv buffer holds the split sort's result
    int split_sort = 1;           // sort the upper halves, then the runs (0: the 8-pass sort)
    DevBuf sort_status;     // onesweep look-back words
    uint32_t sort_epoch = 0;
    DevBuf d_ctl;           // SortCtl
    DevBuf d_box;           // BoxD
    DevBuf d_err;           // uint32 error word
    BoxD box{};             // host copy
    LevelGeom geom{};       // host copy

    // tree
    DevBuf offsets;  // u32, n_total + 1
    DevBuf ranges;   // uint2 (first, last) per node
    DevBuf centers;  // 3 x f64 per node (AoS)
    DevBuf frontier; // build scratch: internal nodes of the current/next level
    DevBuf masks;    // build scratch: ballots of internal children
    DevBuf parts;    // build scratch: per-block counts
    DevBuf d_build;  // BuildCtl
    uint32_t node_capacity = 0;
    uint32_t n_total = 0, n_internal = 0, n_leaf = 0, max_depth_seen = 0;

    // query scratch
    DevBuf q_centers, q_radii, q_counts, q_offsets, q_out, q_out2, q_scan_tmp;
    // query ordering (packet searches): keys, order, look-back words, histograms
    DevBuf qs_keys, qs_keys_alt, qs_ord, qs_ord_alt, qs_status, qs_ctl;
    uint32_t qs_epoch = 0;
    DevBuf packet_ctr;  // dynamic packet counters
    DevBuf knn_fb;      // group kNN: fallback count (u64) at 0, fallback query list (u32) from byte 16
    DevBuf knn_heads;   // group kNN: the heads' largest k-th distances (f64 per head)
    DevBuf stats;       // device counters: points tested, FP64 band re-tests, ...
    // FP32 leaf-relative coordinates (x, y, z, 0) per sorted point, built on demand
    DevBuf rel;
    bool rel_built = false;
    DevBuf crel;  // FP32 (x, y, z) - box centre per point, for the group kNN's FP32 filter
    bool crel_built = false;
    // search configuration (oct_set_search_config)
    int packet = 1;
    int fp32_filter = 0;  // 0, OCT_FP32_ALL, OCT_FP32_RADIUS or OCT_FP32_KNN
    int knn_packet = 1;  // kNN (k <= 64, packet path): groups of queries per warp
    uint32_t knn_bucket = 256;
    int two_pass = 0;   // 1: packet radius searches count, then fill (no result chunks)
    // neighborsStruct searches of the current call: 0, or neighborsApprox's precisionLevel + 1
    // (children deeper than that level are cut; approx_upper adds their ranges)
    uint32_t approx_cut = 0;
    int approx_upper = 0;
    // per-axis radii of the current call (the Vector-radii overloads, cube and square): device pointer to
    // nq x 3 half extents (axes_stride 3) or one (x, y, z) for every query (axes_stride 0); nullptr otherwise
    const double* axes = nullptr;
    uint32_t axes_stride = 0;
    DevBuf q_axes;
    double knn_est = kKnnEstimate;  // register kNN: provisional-threshold factor (0: off)
    uint32_t knn_chunk = kKnnGroupChunk;  // group kNN: consecutive groups per warp fetch
    // one-pass radius search: result chunk pool, links, first chunk per query, counter
    DevBuf ck_pool, ck_next, ck_first, ck_ctr;
    uint32_t ck_cap = 0;

    // pinned host staging for small readbacks
    void* pinned = nullptr;

    // oct_search_timing: CUDA events on the cloud's stream around the main search kernel of each call
    // (kind 0: the packet radius search, 1: the group kNN), summed by oct_search_kernel_times
    bool time_kernels = false;
    std::vector<cudaEvent_t> ev_free;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pend[2];
    double kernel_ms[2] = {0.0, 0.0};
    uint64_t kernel_launches[2] = {0, 0};
};

// Records the start of a timed kernel on the cloud's stream (no-op unless timing is on); stop() records the end.
struct KernelClock {
    Cloud& c;
    int kind;
    cudaEvent_t a = nullptr, b = nullptr;
    KernelClock(Cloud& cl, int k) : c(cl), kind(k) {
        if (!c.time_kernels) return;
        for (cudaEvent_t* e : {&a, &b}) {
            if (!c.ev_free.empty()) {
                *e = c.ev_free.back();
                c.ev_free.pop_back();
            } else if (cudaEventCreate(e) != cudaSuccess) {
                *e = nullptr;
            }
        }
        if (a && b) cudaEventRecord(a, c.stream);
    }
    void stop() {
        if (a && b) {
            cudaEventRecord(b, c.stream);
            c.ev_pend[kind].emplace_back(a, b);
        } else {
            if (a) c.ev_free.push_back(a);
            if (b) c.ev_free.push_back(b);
        }
        a = b = nullptr;
    }
};

// ---- launchers (each returns a cudaError_t of the launch) ----
// upper_hist_only: the split sort follows (the lower digits' histograms are not needed)
cudaError_t launch_bbox_encode(Cloud& c, const double* d_xyz_aos, bool upper_hist_only = false);
cudaError_t launch_sort_split(Cloud& c, const uint32_t skip[8], const double* d_xyz_aos, int* out_sel);
cudaError_t launch_sort_long(Cloud& c, const double* d_xyz_aos, uint32_t l_count, uint32_t l_total);
cudaError_t launch_sort_passes(Cloud& c, const uint32_t skip[8], int* final_sel);
cudaError_t launch_gather(Cloud& c, const double* d_xyz_aos, const uint32_t* d_perm, int sel);
cudaError_t launch_build(Cloud& c, bool* capacity_ok);
cudaError_t launch_radius(Cloud& c, int kernel, int algo, int group, bool fill, const double* d_centers,
                          uint64_t nq, const double* d_radii, double radius, unsigned long long* d_counts,
                          unsigned long long* d_counts2, const unsigned long long* d_offsets, uint32_t* d_out,
                          uint64_t out_capacity);
cudaError_t launch_scan_u64(Cloud& c, const unsigned long long* d_in, unsigned long long* d_out, uint64_t n);
cudaError_t launch_query_order(Cloud& c, const double* d_centers, uint64_t nq, const uint32_t** d_order);
cudaError_t launch_leaf_rel(Cloud& c);
// FP32 coordinates relative to the box centre (group kNN FP32 filter), into c.crel.
cudaError_t launch_center_rel(Cloud& c);
struct ChunkArgs;
// mode as launch_radius_table (0 count, 1 fill, 2 one pass into `chunks`)
cudaError_t launch_radius_packet(Cloud& c, int kernel, int algo, int mode, bool fp32, const double* d_centers,
                                 uint64_t nq, const double* d_radii, double radius, const uint32_t* d_order,
                                 unsigned long long* d_counts, unsigned long long* d_counts2,
                                 const unsigned long long* d_offsets, uint32_t* d_out, uint64_t out_capacity,
                                 const ChunkArgs* chunks = nullptr);
// Result chunks of the one-pass radius search: `cap` chunks of 64 entries, the
// next-chunk links, each query's first chunk, and the hand-out counter.
struct ChunkArgs {
    uint32_t* pool;
    uint32_t* next;
    uint32_t* first;
    uint32_t* ctr;
    uint32_t cap;
};
constexpr uint32_t kResultChunk = 64;

// Packet radius search.  Either one request (`single`, host copy, `packets`
// packets) or the group of a batch (`d_grp`, sizes read on the device); with
// both, every request of the group is on the cloud `single->cv` (kernel
// parameters instead of per-request views).
// mode: 0 count, 1 fill at d_offsets, 2 one pass into `chunks` (counts and
// first chunks written; neighbors / neighborsPrune, FP64 only).
cudaError_t launch_radius_table(int device, cudaStream_t s, int kernel, int algo, int mode, bool fp32,
                                const DynGroup* d_grp, const SearchReq* single, uint64_t packets,
                                const uint32_t* d_order, unsigned long long* d_counts, unsigned long long* d_counts2,
                                const unsigned long long* d_offsets, uint32_t* d_out, uint64_t out_capacity,
                                uint32_t* d_packet_ctr, unsigned long long* d_stats, uint32_t* d_err,
                                int blocks_per_sm = 0, const ChunkArgs* chunks = nullptr);
// Chains of result chunks into CSR (after the counts are scanned into d_offsets).
// Per query, the sum of splitmix64's output function over its result chain.
cudaError_t launch_chunk_hash(int device, cudaStream_t s, const unsigned long long* d_counts, const ChunkArgs& chunks,
                              unsigned long long* d_hashes, uint64_t n, uint32_t* d_err);
cudaError_t launch_chunk_compact(int device, cudaStream_t s, const unsigned long long* d_counts,
                                 const unsigned long long* d_offsets, const ChunkArgs& chunks, uint32_t* d_out,
                                 uint64_t out_capacity, uint64_t n, const uint64_t* d_n, uint32_t* d_err);
// kNN, one warp per query.  Either one request (`single`, nq queries, k <= 64,
// register lists) or the group of a batch (`d_grp`, kmax = the group's largest
// k: register lists up to 64, shared-memory lists up to 1024).
cudaError_t launch_knn_table(int device, cudaStream_t s, const DynGroup* d_grp, const SearchReq* single, uint64_t nq,
                             uint32_t kmax, const uint32_t* d_order, uint32_t bucket, uint32_t* d_idx, double* d_d2,
                             uint32_t* d_counts, uint32_t* d_err, int blocks_per_sm = 0, double est = 0.0);
// Group kNN of a batch group (kmax <= 64: kKnnGroupQueries curve-ordered queries per warp),
// then the per-query kernel over the queries it hands back.  d_fb: the
// fallback group (requests, kmax and q_begin of d_grp, nq = 0 before the
// launch); d_fb_list: one entry per query position of the batch; d_packet_ctr:
// two counters; blocks_per_sm > 0 caps the resident blocks of both launches.
cudaError_t launch_knn_group_table(int device, cudaStream_t s, const DynGroup* d_grp, DynGroup* d_fb,
                                   const SearchReq* single, uint32_t kmax, const uint32_t* d_order, uint32_t bucket,
                                   uint32_t* d_idx, double* d_d2, uint32_t* d_counts, uint32_t* d_err,
                                   uint32_t* d_packet_ctr, uint32_t* d_fb_list, double est, uint32_t chunk,
                                   int blocks_per_sm, double* d_head_kth, size_t head_bytes, bool fp32,
                                   unsigned long long* d_stats);
CloudView cloud_view(const Cloud& c);
// Batched engine: the sort of query keys with device-side sizes (encode_sort.cu),
// and the shared-memory limits of the table kNN list kernels (knn_search.cu).
cudaError_t prepare_sort_dyn();
cudaError_t prepare_knn_dyn();
size_t sort_tile_keys();
cudaError_t launch_sort_dyn(int device, cudaStream_t s, uint64_t* k0, uint64_t* k1, uint32_t* v0, uint32_t* v1,
                            const uint64_t* d_n, uint64_t max_n, int passes, SortCtl* ctl,
                            unsigned long long* status, const uint32_t* d_epoch, uint32_t* err,
                            uint32_t** result_vals);
cudaError_t launch_knn(Cloud& c, const double* d_centers, uint64_t nq, uint32_t k, uint32_t* d_idx, double* d_d2,
                       uint32_t* d_counts);

// oct_search_config.fp32_filter: which searches run their FP32 filter.
inline bool fp32_on_radius(int f) { return f == OCT_FP32_ALL || f == OCT_FP32_RADIUS; }
inline bool fp32_on_knn(int f) { return f == OCT_FP32_ALL || f == OCT_FP32_KNN; }

// One kernel of each source file's device code (each file is its own device
// library), and the loading of every kernel of those libraries on a device
// (capi.cu).  Under lazy module loading, the CUDA default, a kernel is loaded
// at its first launch and the load can wait for the work in flight on the
// device; a server meeting a kernel variant for the first time mid-stream
// would hold its batches that long.  preload_kernels loads them all once per
// device up front.
const void* kernel_anchor_capi();
const void* kernel_anchor_encode_sort();
const void* kernel_anchor_engine();
const void* kernel_anchor_knn_search();
const void* kernel_anchor_octree_build();
const void* kernel_anchor_radius_packet();
const void* kernel_anchor_radius_search();
int preload_kernels(int device);

}  // namespace octb

// The object behind the ABI's oct_cloud handle.
struct oct_cloud_s {
    octb::Cloud c;
};
