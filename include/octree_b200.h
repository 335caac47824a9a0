/*
 * octree_b200.h - C ABI of the B200 linear-octree neighbour search.
 *
 * A drop-in device implementation of the point-cloud neighbour-search path of
 * derivada/octrees-benchmark: Morton/Hilbert 63-bit SFC keys, a stable key sort
 * that reorders the points, the cornerstone linear octree, radius search with
 * the sphere / cube / square / circle kernels through neighbors,
 * neighborsPrune and neighborsStruct, and kNN.  Results are bitwise those of
 * the reference: the same keys, sort order and octree arrays, the same
 * neighbour index sets, and the same kNN squared distances (ties at the k-th
 * distance resolved by the lowest point index).
 *
 * The reference has no FFI; its interface is the C++ template API that these
 * entry points replace (file:line in the reference tree is given per function).
 * A header-only C++ wrapper with the reference's method names sits on top of
 * this ABI (include/linear_octree_gpu.hpp).
 *
 * Conventions
 *  - Every function returns an oct_status; none exits or throws.
 *  - Points and query centres are xyz triples of doubles (AoS, 3 per point).
 *  - Point indices returned by searches index the SFC-sorted cloud, as in the
 *    reference (the points are reordered in place by sortPoints).
 *  - Buffers are host memory unless OCT_MEM_DEVICE is passed, in which case
 *    every pointer argument of that call is device memory of the cloud's
 *    device; host-memory calls synchronise the cloud's stream before they
 *    return, device-memory calls that do not need a readback return without
 *    waiting.
 *  - One cloud is used by one host thread at a time; different clouds are
 *    independent and may be used concurrently.
 */
#ifndef OCTREE_B200_H
#define OCTREE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OCT_ABI_VERSION 1

typedef enum {
    OCT_OK = 0,
    OCT_ERR_INVALID_ARG = 1,   /* bad pointer, size, enum value */
    OCT_ERR_CUDA = 2,          /* a CUDA call failed (see oct_last_error) */
    OCT_ERR_OUT_OF_MEMORY = 3, /* a device allocation failed */
    OCT_ERR_STATE = 4,         /* call out of order (e.g. search before build) */
    OCT_ERR_CAPACITY = 5,      /* caller's output buffer too small; the needed size is returned */
    OCT_ERR_DEVICE_LIMIT = 6,  /* a bounded device loop hit its limit (stack, spin) */
    OCT_ERR_NO_DEVICE = 7      /* no usable CUDA device */
} oct_status;

/* Encoders: the reference's EncoderType values (inc/main_options.hpp:73-83). */
typedef enum { OCT_ENC_MORTON_3D = 1, OCT_ENC_HILBERT_3D = 5 } oct_encoder;

/* Search kernels: the reference's Kernel_t values (inc/main_options.hpp:97-103). */
typedef enum { OCT_KERNEL_CIRCLE = 0, OCT_KERNEL_SPHERE = 1, OCT_KERNEL_SQUARE = 2, OCT_KERNEL_CUBE = 3 } oct_kernel;

/* Radius-search variants of LinearOctree (inc/structures/linear_octree.hpp):
 * neighbors 796-816, neighborsPrune 746-784, neighborsStruct 695-736,
 * neighborsApprox 975-1035 (oct_approx_search); the values of the reference's
 * SearchAlgo (inc/main_options.hpp:29-35). */
typedef enum {
    OCT_NEIGHBORS = 1,
    OCT_NEIGHBORS_PRUNE = 2,
    OCT_NEIGHBORS_STRUCT = 3,
    OCT_NEIGHBORS_APPROX = 4
} oct_algo;

#define OCT_MEM_DEVICE 0x1u /* every buffer of the call is device memory */

/* oct_params.flags: sort with eight 8-bit passes over the whole keys instead of
 * four passes over their upper halves followed by the runs of equal upper
 * halves (same result; the split sort is the default and takes the 8-pass
 * sort by itself when a run is longer than 4096 points) */
#define OCT_CLOUD_SORT_8PASS 0x1u

typedef struct {
    uint32_t max_points_leaf; /* mainOptions.maxPointsLeaf (main_options.hpp:210); default 128 */
    int32_t encoder;          /* oct_encoder */
    int32_t device;           /* CUDA device ordinal */
    uint32_t flags;           /* OCT_CLOUD_* */
} oct_params;

typedef struct {
    uint64_t n_points;
    uint32_t n_leaf;         /* LinearOctree::nLeaf */
    uint32_t n_internal;     /* LinearOctree::nInternal = (nLeaf - 1) / 7 */
    uint32_t n_total;        /* LinearOctree::nTotal */
    uint32_t max_depth_seen; /* LinearOctree::maxDepthSeen */
} oct_tree_info;

typedef struct oct_cloud_s* oct_cloud;

/* Library version (OCT_ABI_VERSION) and a static description of a status. */
int oct_abi_version(void);
const char* oct_status_string(int status);

/* Create / destroy a device-resident cloud.  Replaces constructing the
 * reference's encoder (getEncoder, inc/encoding/point_encoder_factory.hpp:12)
 * and setting mainOptions.maxPointsLeaf; nothing global is read. */
int oct_cloud_create(const oct_params* params, oct_cloud* out);
int oct_cloud_destroy(oct_cloud cloud);

/* Run the cloud's work on this CUDA stream (cudaStream_t) instead of its own. */
int oct_cloud_set_stream(oct_cloud cloud, void* cuda_stream);

/* Last error message of the cloud (NUL-terminated, truncated to len). */
int oct_last_error(oct_cloud cloud, char* buf, size_t len);

/* Wait for the cloud's queued device work and report an error latched by a
 * device-memory call that returned before its kernels ran.  No reference
 * counterpart (the reference is synchronous). */
int oct_synchronize(oct_cloud cloud);

/* Lanes per query of the radius traversal: 8, 16 or 32 (4, 2 or 1 queries per
 * warp); other values select the default (8).  No reference counterpart: the
 * autotuner sets it. */
int oct_set_radius_group(oct_cloud cloud, int lanes);

/* Search configuration of a cloud (no reference counterpart; set by the
 * autotuner or the caller).  Results are identical in every configuration.
 *  packet       1 (default): the query centres are ordered along the cloud's
 *               curve and each warp walks the tree once for 32 neighbouring
 *               queries; 0: one query per group of radius_lanes lanes.
 *  fp32_filter  OCT_FP32_ALL (1): radius searches test leaf points in FP32
 *               relative to their leaf's centre and re-test in FP64 only points
 *               within a rigorous error band of the boundary (packet path); the
 *               group kNN (knn_packet, k <= 64) tests points in FP32 relative
 *               to the box centre and computes the exact FP64 distance only for
 *               points within a rigorous band of the query's k-th distance or
 *               inside it.  OCT_FP32_RADIUS (2): the radius filter only;
 *               OCT_FP32_KNN (3): the kNN filter only; 0 (default): every test
 *               in FP64.  Results are the same.
 *  radius_lanes lanes per query when packet is 0: 8 (default), 16 or 32.
 *  knn_packet   1 (default): kNN with k <= 64 on the packet path walks the
 *               tree once per group of 4 curve-ordered queries per warp
 *               (queries whose provisional threshold turns out too small
 *               finish on the per-query kernel); 0: one warp per query,
 *               visited in curve order when packet is 1.
 *  knn_bucket   kNN with k <= 64 on the packet path scans any subtree of at
 *               most this many points as one contiguous range instead of
 *               descending into it (default 256; 0 descends to the leaves).
 *               Extra points cannot change the k best pairs.
 *  reserved[0]  1: packet radius searches count, then fill at the scanned
 *               offsets; 0 (default): one pass into per-query result chunks.
 *  reserved[1]  kNN (k <= 64, packet path) provisional threshold, in percent of
 *               the radius holding k points at the density of the query's first
 *               cell: 0 = the default (120), < 0 = off.  Results are the same.
 *  reserved[2]  knn_packet: consecutive query groups a warp takes at a time
 *               (1-64; 0 = the default); every group after the first of a
 *               run starts from the previous group's k-th distances.  Results
 *               are the same. */
#define OCT_FP32_ALL 1    /* oct_search_config.fp32_filter: radius and kNN FP32 filters */
#define OCT_FP32_RADIUS 2 /* the radius filter only */
#define OCT_FP32_KNN 3    /* the kNN filter only */
typedef struct {
    int32_t packet;
    int32_t fp32_filter;
    int32_t radius_lanes;
    int32_t knn_packet;
    int32_t knn_bucket;
    int32_t reserved[3];
} oct_search_config;
int oct_set_search_config(oct_cloud cloud, const oct_search_config* config);

/* Counters of the packet radius searches since the last reset: point tests
 * and FP64 re-tests of points inside the FP32 error band (the band-hit
 * fraction is their ratio).  Waits for the cloud's stream. */
int oct_search_stats(oct_cloud cloud, uint64_t* point_tests, uint64_t* fp64_retests, int reset);
/* Counters of the group kNN's FP32 filter (k <= 64, packet path, fp32_filter
 * on) since the last reset: point tests made in FP32, those that went on to the
 * exact FP64 distance (the candidates and the band), and band hits (FP64 tests
 * whose point then failed the exact test: the filter's only extra work).  No
 * reference counterpart. */
int oct_knn_filter_stats(oct_cloud cloud, uint64_t* point_tests, uint64_t* fp64_tests, uint64_t* band_hits,
                         int reset);

/* Device timing of the main search kernel of each call on this cloud: with
 * timing on, CUDA events on the cloud's stream bracket the packet radius
 * kernel (k_radius_packet) and the group kNN kernel (k_knn_group) of every
 * call; oct_search_kernel_times waits for the stream and returns the summed
 * milliseconds and launch counts since the last reset (any pointer may be
 * NULL).  For roofline measurements; no reference counterpart. */
int oct_search_timing(oct_cloud cloud, int enable);
int oct_search_kernel_times(oct_cloud cloud, double* radius_ms, uint64_t* radius_launches, double* knn_ms,
                            uint64_t* knn_launches, int reset);

/* Upload n points (xyz AoS).  Replaces filling the reference's PointsAoS
 * container (inc/geometry/point_containers.hpp:32-65). */
int oct_set_points(oct_cloud cloud, const double* xyz, uint64_t n, uint32_t flags);

/* Bounding box, SFC keys, stable key sort and point reorder.  Replaces
 * PointEncoder::sortPoints(points, meta) (inc/encoding/point_encoder.hpp:484-503):
 * box12 (center xyz, radii xyz, min xyz, max xyz of the returned Box),
 * keys (n sorted keys), perm (n: input position of each sorted point, the
 * reference's Point::id), sorted_xyz (n x 3, the reordered points).  Any
 * output may be NULL. */
int oct_encode_sort(oct_cloud cloud, double* box12, uint64_t* keys, uint32_t* perm, double* sorted_xyz,
                    uint32_t flags);

/* A cloud that is already sorted: n points (xyz AoS) in curve order with
 * their ascending 63-bit codes and the Box they were encoded in (box12:
 * center, radii, min, max, as oct_encode_sort returns it).  This is the input
 * of the reference's LinearOctree(points, codes, box, enc) constructor
 * (inc/structures/linear_octree.hpp:614-623) when sortPoints ran separately;
 * oct_build follows.  The points are taken in the order given (perm is the
 * identity); host codes are checked to be ascending and below 2^63, device
 * codes (OCT_MEM_DEVICE) are not. */
int oct_set_sorted_points(oct_cloud cloud, const double* sorted_xyz, const uint64_t* keys, uint64_t n,
                          const double* box12, uint32_t flags);

/* Build the linear octree over the sorted cloud.  Replaces the
 * LinearOctree(points, codes, box, enc) constructor
 * (inc/structures/linear_octree.hpp:614-623, buildOctree 567-605). */
int oct_build(oct_cloud cloud, oct_tree_info* info);

/* Export the built tree: offsets (n_total + 1, first child or 0 for a leaf),
 * ranges (n_total x 2: first, last point), centers (n_total x 3), radii
 * (22 x 3, precomputedRadii), half (3, halfLengths).  Any output may be NULL.
 * The arrays are LinearOctree's members of the same names
 * (linear_octree.hpp:112-121, 140). */
int oct_tree_export(oct_cloud cloud, uint32_t* offsets, uint64_t* ranges, double* centers, double* radii,
                    double* half, uint32_t flags);

/* Restore a sorted and built cloud from a checkpoint, without sorting or
 * building: info, box12, keys, perm and sorted_xyz as oct_build and
 * oct_encode_sort returned them, offsets (n_total; the trailing 0 is not
 * needed), ranges, centers, radii and half as oct_tree_export returned them.
 * The reference has no counterpart (it rebuilds from the points each run); the
 * arrays are its LinearOctree members (linear_octree.hpp:112-121, 140).  The
 * cloud must have been created with the checkpoint's encoder and leaf size.
 * Host buffers only (flags 0).  The arrays are checked (counts, ascending
 * keys, a permutation, offsets and ranges in bounds) and OCT_ERR_INVALID_ARG
 * names the first violation; the cloud then answers every search as the
 * original did. */
int oct_tree_import(oct_cloud cloud, const oct_tree_info* info, const double* box12, const uint64_t* keys,
                    const uint32_t* perm, const double* sorted_xyz, const uint32_t* offsets, const uint64_t* ranges,
                    const double* centers, const double* radii, const double* half, uint32_t flags);

/* Radius search for nq centres (xyz AoS).  radii: per-query radii (nq
 * doubles) or NULL to use `radius` for every query.
 * Replaces neighbors / neighborsPrune (linear_octree.hpp:1050-1087): the
 * result is CSR, offsets (nq + 1) and point indices (offsets[nq] of them, each
 * query's ascending).  If idx_capacity is smaller than the total, offsets and
 * *total are still written and OCT_ERR_CAPACITY is returned.  For
 * OCT_NEIGHBORS_STRUCT the indices are those of the expanded ranges. */
int oct_radius_search(oct_cloud cloud, int kernel, int algo, const double* centers, uint64_t nq,
                      const double* radii, double radius, uint64_t* offsets, uint32_t* idx, uint64_t idx_capacity,
                      uint64_t* total, uint32_t flags);

/* Neighbour counts only (the size() of each result), per query. */
int oct_radius_count(oct_cloud cloud, int kernel, int algo, const double* centers, uint64_t nq, const double* radii,
                     double radius, uint64_t* counts, uint32_t flags);

/* Neighbour counts and an order-independent hash of each neighbour set, per
 * query, without the neighbour lists (for sweeps whose lists would not fit
 * anywhere, e.g. every point of a large cloud as a centre, and for checking
 * sets against another implementation): hashes[q] = sum over the neighbours i
 * of splitmix64's output function of i, modulo 2^64 (z = i + 0x9E3779B97F4A7C15;
 * z = (z ^ z >> 30) * 0xBF58476D1CE4E5B9; z = (z ^ z >> 27) * 0x94D049BB133111EB;
 * z ^ z >> 31).  Sets as oct_radius_search (OCT_NEIGHBORS_STRUCT: the expanded
 * ranges).  counts and hashes: nq entries each. */
int oct_radius_hash(oct_cloud cloud, int kernel, int algo, const double* centers, uint64_t nq, const double* radii,
                    double radius, uint64_t* counts, uint64_t* hashes, uint32_t flags);

/* neighborsStruct ranges (linear_octree.hpp:1038-1042, NeighborSet
 * neighbor_set.hpp:16-90): CSR over half-open ranges, range_offsets (nq + 1)
 * and pairs (first, last) in ascending order, exactly the ranges the reference
 * adds (one per fully-inside node, including empty ones, and each maximal run
 * of inside points of a leaf); point_counts (nq, may be NULL) is
 * NeighborSet::numberOfPoints.  Capacity handling as oct_radius_search. */
int oct_struct_search(oct_cloud cloud, int kernel, const double* centers, uint64_t nq, const double* radii,
                      double radius, uint64_t* range_offsets, uint32_t* pairs, uint64_t pair_capacity,
                      uint64_t* total_ranges, uint64_t* point_counts, uint32_t flags);

/* The Vector-radii overloads of neighbors / neighborsPrune / neighborsStruct
 * (linear_octree.hpp:1044-1048, 1056-1060, 1069-1074; kernelFactory(center,
 * Vector), kernels/kernel_factory.hpp:33-41): the kernel's box is
 * centre -/+ (rx, ry, rz).  Square and cube kernels only (the reference's
 * static_assert); other kernels are rejected with OCT_ERR_INVALID_ARG.
 * radii_xyz: nq x 3 half extents when per_query is non-zero, else one (x, y, z)
 * for every query (the same buffer kind as the centres: host, or device with
 * OCT_MEM_DEVICE).  Outputs and capacity handling as oct_radius_search /
 * oct_struct_search.  These calls run the group-per-query search path whatever
 * the cloud's search configuration. */
int oct_radius_search_axes(oct_cloud cloud, int kernel, int algo, const double* centers, uint64_t nq,
                           const double* radii_xyz, int per_query, uint64_t* offsets, uint32_t* idx,
                           uint64_t idx_capacity, uint64_t* total, uint32_t flags);
int oct_struct_search_axes(oct_cloud cloud, int kernel, const double* centers, uint64_t nq, const double* radii_xyz,
                           int per_query, uint64_t* range_offsets, uint32_t* pairs, uint64_t pair_capacity,
                           uint64_t* total_ranges, uint64_t* point_counts, uint32_t flags);

/* neighborsApprox (linear_octree.hpp:975-1035): the neighborsStruct search cut
 * below depth precision_level.  A child deeper than that level is not judged:
 * with upper_bound its whole range is added (every octant whose parent the
 * search reached, so the points are a superset of the exact set), without it
 * the child is dropped (a subset).  Outputs and capacity handling as
 * oct_struct_search; the ranges are the reference's, in ascending order.  The
 * reference's Point overloads (1089-1111) pass their tolerance percentage on as
 * the precision level (converted to an unsigned integer): the same level here.
 * A level of 21 or more cuts nothing (the neighborsStruct result). */
int oct_approx_search(oct_cloud cloud, int kernel, const double* centers, uint64_t nq, const double* radii,
                      double radius, uint32_t precision_level, int upper_bound, uint64_t* range_offsets,
                      uint32_t* pairs, uint64_t pair_capacity, uint64_t* total_ranges, uint64_t* point_counts,
                      uint32_t flags);

/* k nearest neighbours of nq centres.  Replaces LinearOctree::knn
 * (linear_octree.hpp:899-942): idx and d2 are nq x k, ascending by squared
 * distance (ties by index); counts[q] = min(n, k); unused slots hold
 * UINT32_MAX / +inf.  counts may be NULL. */
int oct_knn(oct_cloud cloud, const double* centers, uint64_t nq, uint32_t k, uint32_t* idx, double* d2,
            uint32_t* counts, uint32_t flags);

/* ---- Batched engine: many clouds and request sets in one launch ----------
 *
 * No reference counterpart: the reference answers one query at a time per
 * OpenMP thread (neighbor_benchmarks.hpp:502-568).  An engine runs a batch of
 * requests (each a set of radius or kNN centres against one built cloud) as
 * one device pass: the centres of every request are ordered along their
 * cloud's curve by one sort, then one persistent launch per kernel variant
 * answers all radius requests (count, scan, fill) while the kNN requests run
 * on a second stream.  Sizes are read on the device, so the launch sequence
 * of a batch shape (which variants occur) is captured once as a CUDA graph
 * and replayed for every later batch of that shape.  Results are bitwise
 * those of the single-cloud calls. */
typedef struct oct_engine_s* oct_engine;

#define OCT_ENGINE_NO_GRAPH 0x1u /* launch the sequence directly instead of through a graph */

typedef struct {
    int32_t device;        /* CUDA device ordinal; clouds of a batch must live there */
    uint32_t flags;        /* OCT_ENGINE_* */
    uint64_t reserve_queries; /* initial capacity hint: centres per batch (0: grow on demand) */
    uint64_t reserve_results; /* initial capacity hint: radius results per batch */
} oct_engine_params;

typedef enum { OCT_REQ_RADIUS = 0, OCT_REQ_KNN = 1 } oct_request_type;

/* One request of a batch.  centers (and radii) are device memory of the
 * engine's device and must stay valid until the batch has completed. */
typedef struct {
    oct_cloud cloud;       /* a built cloud */
    int32_t type;          /* oct_request_type */
    int32_t kernel;        /* radius: oct_kernel */
    int32_t algo;          /* radius: OCT_NEIGHBORS or OCT_NEIGHBORS_PRUNE */
    uint32_t k;            /* kNN: 1..1024 */
    const double* centers; /* nq x 3 */
    uint64_t nq;
    const double* radii;   /* radius: nq per-centre radii, or NULL to use `radius` */
    double radius;
} oct_request;

/* Where a request's results are in the engine's output arrays
 * (oct_engine_outputs).  Radius: offsets[q_begin .. q_begin + nq] index the
 * indices array (each centre's neighbours ascending).  kNN: rows of k slots
 * from out_begin in knn_idx / knn_d2 (nq x k), counts at knn_counts[q_begin +
 * i]. */
typedef struct {
    uint64_t q_begin;
    uint64_t out_begin;
    uint64_t nq;
    uint64_t n_results;    /* radius: neighbours of the request (after completion) */
} oct_request_place;

int oct_engine_create(const oct_engine_params* params, oct_engine* out);
int oct_engine_destroy(oct_engine engine);
/* Run on this CUDA stream (cudaStream_t); kNN work forks onto a private stream and joins back. */
int oct_engine_set_stream(oct_engine engine, void* cuda_stream);
int oct_engine_last_error(oct_engine engine, char* buf, size_t len);
/* Search configuration of the engine (oct_search_config: fp32_filter (0-3, as for
 * a cloud), knn_bucket;
 * knn_packet = 1 (the engine's default): kNN with k <= 64 in groups of 4
 * curve-ordered queries per warp, 0: one warp per query;
 * reserved[0] = radius blocks per SM, reserved[1] = kNN blocks per SM, 0 = default;
 * reserved[2] = 1 to run kNN after the radius search instead of beside it). */
int oct_engine_set_config(oct_engine engine, const oct_search_config* config);
int oct_engine_get_config(oct_engine engine, oct_search_config* config);

/* Enqueue a batch (returns without waiting); places (n entries, may be NULL
 * until oct_engine_wait) receive each request's output position.  One batch
 * is in flight per engine: a second submit waits for the first. */
int oct_engine_submit(oct_engine engine, const oct_request* requests, uint32_t n, oct_request_place* places);
/* Wait for the submitted batch; grows the result array and re-runs the batch
 * when its results did not fit.  radius_total (may be NULL) = all radius
 * results of the batch; places as in submit, with n_results filled in. */
int oct_engine_wait(oct_engine engine, oct_request_place* places, uint64_t* radius_total);
/* submit + wait. */
int oct_engine_run(oct_engine engine, const oct_request* requests, uint32_t n, oct_request_place* places,
                   uint64_t* radius_total);
/* Device pointers of the output arrays of the last completed batch (valid until the next submit). */
int oct_engine_outputs(oct_engine engine, uint64_t** offsets, uint32_t** indices, uint32_t** knn_idx,
                       double** knn_d2, uint32_t** knn_counts);
/* A radius request's per-centre neighbour counts and set hashes (as
 * oct_radius_hash), computed on the device from the batch's results: 16 bytes
 * per centre cross to the host instead of the lists.  counts and hashes: nq
 * entries each (host buffers, or device buffers with OCT_MEM_DEVICE). */
int oct_engine_copy_radius_hash(oct_engine engine, const oct_request_place* place, uint64_t* counts,
                                uint64_t* hashes, uint32_t flags);
/* Copy one request's results out (host memory unless flags has OCT_MEM_DEVICE).
 * Radius: offsets (nq + 1, rebased to 0) and idx (up to idx_capacity).  kNN:
 * idx, d2 (nq x k) and counts (nq); any may be NULL. */
int oct_engine_copy_radius(oct_engine engine, const oct_request_place* place, uint64_t* offsets, uint32_t* idx,
                           uint64_t idx_capacity, uint32_t flags);
int oct_engine_copy_knn(oct_engine engine, const oct_request_place* place, uint32_t k, uint32_t* idx, double* d2,
                        uint32_t* counts, uint32_t flags);
/* Time the candidate configurations (FP32 filter, blocks per SM, kNN bucket)
 * on a sample batch and keep the fastest; *chosen (may be NULL) receives it.
 * Results do not depend on the configuration. */
int oct_engine_autotune(oct_engine engine, const oct_request* requests, uint32_t n, oct_search_config* chosen);
/* Device time (ms) of the last completed batch, from events around its launch sequence. */
int oct_engine_last_ms(oct_engine engine, float* ms);
/* *ready = 1 when the submitted batch has finished on the device (oct_engine_wait will not block). */
int oct_engine_ready(oct_engine engine, int* ready);
/* Device bytes the engine's arrays hold. */
int oct_engine_memory(oct_engine engine, uint64_t* bytes);
/* Device bytes a cloud holds (points, keys, tree, search scratch). */
int oct_cloud_memory(oct_cloud cloud, uint64_t* bytes);

/* Health check of the bounded device waits.  Launches one kernel on `device`
 * that waits for a device flag nothing sets, the way the library's cross-block
 * waits wait (poll, back off, give up after spin_limit polls; 0 = the library's
 * own limit, 2^26 polls, a few seconds), and reads its status back.  Returns
 * OCT_ERR_DEVICE_LIMIT when the wait ran out, as it must, with *polls (may be
 * NULL) the polls it made; the device stays usable.  OCT_OK would mean the
 * flag was seen set. */
int oct_device_wait_probe(int device, uint32_t spin_limit, uint32_t* polls);

/* Clouds take their device arrays from one stream-ordered pool per device,
 * which keeps what destroyed clouds free for the next clouds (returning it to
 * the driver would make other threads' CUDA calls wait).  This returns the
 * pool's unused memory to the driver. */
int oct_trim_cloud_memory(int device);

/* ---- Serving: continuous batching over device-resident clouds ------------
 *
 * No reference counterpart.  A server owns `slots` engines, each on its own
 * stream.  Clients submit requests from any thread; a scheduler thread forms a
 * batch from the queue whenever a slot is free - smallest expected work first,
 * a request waiting longer than max_wait_ms first of all (OCT_SERVER_FIFO:
 * arrival order) - admitting requests while the registered clouds, the
 * batches in flight and the new batch fit the HBM budget (a request that does
 * not fit waits: an admission stall), and launches it.  Batches on different slots overlap on the device.
 * A completed request's results stay in its slot until the client releases
 * the ticket; a slot is reused once all its tickets are released.  With
 * OCT_SERVER_PLAIN the server instead runs one request per launch through the
 * single-cloud path, first come first served (the baseline). */
typedef struct oct_server_s* oct_server;

#define OCT_SERVER_PLAIN 0x1u /* one request per launch, single-cloud plain path */
#define OCT_SERVER_FIFO 0x2u  /* batched: admit in arrival order only (no smallest-first admission) */
#define OCT_SERVER_NO_GRAPH 0x4u /* batched: launch each batch's kernels directly, not from captured graphs */
#define OCT_CLOUD_OWNED 0x1u  /* oct_server_add_cloud: the server destroys the cloud when it evicts or removes it */

typedef struct {
    int32_t device;
    uint32_t flags;              /* OCT_SERVER_* */
    uint32_t slots;              /* batches in flight at once; 0: 3 */
    uint32_t max_batch_requests; /* 0: 1024 */
    uint64_t max_batch_queries;  /* 0: 512K */
    uint64_t hbm_budget;         /* bytes for the clouds and the admitted batches; 0: 120 GB */
    double max_wait_ms;          /* requests queued longer than this are admitted first, in arrival
                                    order; the others smallest estimated work first; 0: 40 ms */
} oct_server_params;

typedef struct {
    uint64_t ticket;
    int32_t status;    /* oct_status of the request */
    int32_t type;      /* oct_request_type */
    uint64_t nq;
    uint64_t n_results; /* radius: neighbours of the request */
    double queue_ms;   /* submit to launch */
    double latency_ms; /* submit to results complete on the device */
} oct_completion;

typedef struct {
    uint64_t submitted, completed, batches, admission_stalls, evictions, queries;
    uint64_t cloud_bytes, inflight_bytes, peak_bytes;
    uint32_t queued, in_flight;
    double max_submit_ms; /* the longest host call that launched a batch (graph capture included) */
    double max_finish_ms; /* the longest host call that completed a batch (result-array growth included) */
} oct_server_stats;

int oct_server_create(const oct_server_params* params, oct_server* out);
int oct_server_destroy(oct_server server);
int oct_server_last_error(oct_server server, char* buf, size_t len);
/* Search configuration of every slot (as oct_engine_set_config). */
int oct_server_set_config(oct_server server, const oct_search_config* config);
/* Register a built cloud (its bytes count against the budget).  When it does
 * not fit, idle clouds added with OCT_CLOUD_OWNED are evicted, least recently
 * used first; OCT_ERR_OUT_OF_MEMORY if that is not enough. */
int oct_server_add_cloud(oct_server server, oct_cloud cloud, uint32_t flags);
/* Unregister a cloud once no queued or running request uses it. */
int oct_server_remove_cloud(oct_server server, oct_cloud cloud);
/* Queue a request on a registered cloud (centres as oct_engine_submit: device
 * memory, valid until the request completes).  For admission, a radius
 * request with per-centre radii should set `radius` to their maximum. */
int oct_server_submit(oct_server server, const oct_request* request, uint64_t* ticket);
/* Completed requests, up to max; waits up to wait_ms for the first one. */
int oct_server_poll(oct_server server, oct_completion* out, uint32_t max, uint32_t* n, int32_t wait_ms);
/* A completed request's results, as oct_engine_copy_radius / oct_engine_copy_knn. */
int oct_server_copy_radius(oct_server server, uint64_t ticket, uint64_t* offsets, uint32_t* idx,
                           uint64_t idx_capacity, uint32_t flags);
int oct_server_copy_knn(oct_server server, uint64_t ticket, uint32_t* idx, double* d2, uint32_t* counts,
                        uint32_t flags);
/* The client is done with a completed request's results. */
int oct_server_release(oct_server server, uint64_t ticket);
int oct_server_get_stats(oct_server server, oct_server_stats* stats);

/* Largest cloud oct_encode_sort_noalloc accepts. */
#define OCT_NOALLOC_MAX_POINTS (1u << 18) /* 262,144 points */

/* Allocation-free bounding box + SFC keys + stable sort, for callers that
 * cannot allocate device memory when they call in: code running inside a
 * memory pool or allocator it does not own, plugin hosts that forbid
 * cudaMalloc / cudaFree on their streams, and latency-bound loops that cannot
 * afford the device-wide synchronisation cudaMalloc / cudaFree cause.  No
 * counterpart in the reference (whose PointEncoder::sortPoints allocates on
 * the host heap); it computes what oct_encode_sort computes, bit for bit.
 *
 * All pointers are device memory of the current CUDA device: d_xyz (n x 3
 * doubles, AoS), d_keys (n sorted keys), d_perm (n input positions of the
 * sorted points) and d_box12 (12 doubles: center, radii, min, max).  The work
 * is queued on `stream` (a cudaStream_t, NULL for the default stream) and the
 * call returns without waiting.  It calls no cudaMalloc, cudaFree or other
 * allocating routine: its scratch is one fixed device array of about 3.2 MB,
 * which every GPU that loads this library holds until the process exits.
 * Limits and rules:
 *  - n above OCT_NOALLOC_MAX_POINTS is rejected with OCT_ERR_INVALID_ARG;
 *  - the first call on a device looks up the scratch array's device address
 *    (once per device, with that device current); make that first call before
 *    any stream capture;
 *  - every call on a device shares the one scratch array and clears what must
 *    start at zero itself, so calls whose work overlaps on the GPU (other
 *    streams, other host threads) race and must be serialised by the caller;
 *  - the address looked up at the first call is kept for the life of the
 *    process: do not call this entry point on a device after cudaDeviceReset
 *    (or after its primary context was released and made again);
 *  - errors found on the device arrive with the results, not in the return
 *    code (the call does not wait): if a sort pass's bounded wait for an
 *    earlier tile gave up, some keys and ids were not written and d_box12's
 *    radii (elements 3..5) hold -1.0, which no Box can hold.  Check them after
 *    synchronising the stream. */
int oct_encode_sort_noalloc(int encoder, const double* d_xyz, uint64_t n, uint64_t* d_keys, uint32_t* d_perm,
                            double* d_box12, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* OCTREE_B200_H */
