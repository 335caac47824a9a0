// The extern "C" boundary (include/octree_b200.h): cloud handles, host/device
// buffer handling, call ordering, and the error word the kernels latch.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <utility>
#include <vector>

#include <mutex>

#include <cudaTypedefs.h>

#include "cloud.h"

using namespace octb;

namespace {

// Makes the cloud's device current for the duration of a call.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int set_error(Cloud& c, int status, const std::string& msg) {
    c.last_error = msg;
    return status;
}

int cuda_fail(Cloud& c, cudaError_t e, const char* what) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
    const int st = (e == cudaErrorMemoryAllocation) ? OCT_ERR_OUT_OF_MEMORY : OCT_ERR_CUDA;
    cudaGetLastError();  // clear a sticky launch error
    return set_error(c, st, buf);
}

#define CK(expr)                                          \
    do {                                                  \
        cudaError_t _e = (expr);                          \
        if (_e != cudaSuccess) return cuda_fail(c, _e, #expr); \
    } while (0)


// Synchronise the stream and turn the latched device error word into a status.
// Pinned staging layout: [0, 2048) readbacks of structs, [2048, 2056) the error word.
constexpr size_t kPinnedErrOffset = 2048;

int sync_and_check(Cloud& c, uint32_t ignore_bits = 0) {
    uint32_t* h = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(c.pinned) + kPinnedErrOffset);
    CK(cudaMemcpyAsync(h, c.d_err.ptr, 4, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    const uint32_t bits = *h & ~ignore_bits;
    if (*h) CK(cudaMemsetAsync(c.d_err.ptr, 0, 4, c.stream));
    if (bits & kErrOutputCapacity) return set_error(c, OCT_ERR_CAPACITY, "output buffer smaller than the results");
    if (bits & kErrBadInput) return set_error(c, OCT_ERR_INVALID_ARG, "device rejected an input");
    if (bits) {
        char buf[128];
        snprintf(buf, sizeof(buf), "a bounded device loop hit its limit (error bits 0x%x)", bits);
        return set_error(c, OCT_ERR_DEVICE_LIMIT, buf);
    }
    return OCT_OK;
}

// Copy a caller buffer to the device when it is host memory; return the device pointer.
template <class T>
int stage_in(Cloud& c, DevBuf& scratch, const T* src, size_t count, bool device, const T** out) {
    if (device || src == nullptr) {
        *out = src;
        return OCT_OK;
    }
    CK(scratch.reserve(sizeof(T) * (count ? count : 1)));
    if (count) CK(cudaMemcpyAsync(scratch.ptr, src, sizeof(T) * count, cudaMemcpyHostToDevice, c.stream));
    *out = scratch.as<T>();
    return OCT_OK;
}

template <class T>
int copy_out(Cloud& c, T* dst, const T* dsrc, size_t count, bool device) {
    if (!dst || count == 0) return OCT_OK;
    CK(cudaMemcpyAsync(dst, dsrc, sizeof(T) * count, device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                       c.stream));
    return OCT_OK;
}

__global__ void k_soa_to_aos(const double* xs, const double* ys, const double* zs, uint64_t n, double* out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        out[3 * i] = xs[i];
        out[3 * i + 1] = ys[i];
        out[3 * i + 2] = zs[i];
    }
}

__global__ void k_widen_pairs(const uint2* in, uint64_t n, unsigned long long* out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const uint2 v = in[i];
        out[2 * i] = v.x;
        out[2 * i + 1] = v.y;
    }
}

__global__ void k_aos_to_soa_iota(const double* xyz, uint64_t n, double* xs, double* ys, double* zs,
                                  uint32_t* perm) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        xs[i] = xyz[3 * i];
        ys[i] = xyz[3 * i + 1];
        zs[i] = xyz[3 * i + 2];
        perm[i] = (uint32_t)i;
    }
}

bool valid_kernel(int k) { return k >= OCT_KERNEL_CIRCLE && k <= OCT_KERNEL_CUBE; }
bool valid_algo(int a) { return a >= OCT_NEIGHBORS && a <= OCT_NEIGHBORS_STRUCT; }

// Count or fill pass of a radius search on the configured path.  With the
// packet path the query order (sorted along the curve) is computed once per
// call by the first pass and reused by the second.
cudaError_t radius_pass(Cloud& c, int kernel, int algo, bool fill, const double* dq, uint64_t nq, const double* dr,
                        double radius, unsigned long long* counts, unsigned long long* counts2,
                        const unsigned long long* offs, uint32_t* out, uint64_t cap, const uint32_t** order) {
    if (!c.packet) return launch_radius(c, kernel, algo, c.radius_group, fill, dq, nq, dr, radius, counts, counts2, offs,
                                        out, cap);
    cudaError_t e;
    if (fp32_on_radius(c.fp32_filter) && !c.rel_built) {
        if ((e = launch_leaf_rel(c)) != cudaSuccess) return e;
        c.rel_built = true;
    }
    if ((e = c.stats.reserve(64)) != cudaSuccess) return e;
    if (!*order && (e = launch_query_order(c, dq, nq, order)) != cudaSuccess) return e;
    return launch_radius_packet(c, kernel, algo, fill ? 1 : 0, fp32_on_radius(c.fp32_filter), dq, nq, dr, radius,
                                *order, counts, counts2, offs, out, cap);
}

// Radius search in one traversal (packet path, FP64 or FP32 filter): every query's results go
// to its chain of result chunks, the counts are scanned, and the chains are
// compacted into the CSR output.  A pool that turned out too small leaves the
// counts exact: it is sized from the total and the traversal runs once more.
int radius_chunks(Cloud& c, int kernel, int algo, const double* dq, uint64_t nq, const double* dr, double radius,
                  unsigned long long* doffs, uint64_t* total) {
    const int pass_algo = (algo == OCT_NEIGHBORS_STRUCT) ? OCT_NEIGHBORS_PRUNE : algo;  // same index set
    unsigned long long* dc = c.q_counts.as<unsigned long long>();
    CK(c.stats.reserve(64));
    CK(c.ck_first.reserve(4 * nq));
    CK(c.ck_ctr.reserve(256));
    const uint32_t* order = nullptr;
    CK(launch_query_order(c, dq, nq, &order));
    if (fp32_on_radius(c.fp32_filter) && !c.rel_built) {  // the FP32 filter reads leaf-relative coordinates
        CK(launch_leaf_rel(c));
        c.rel_built = true;
    }
    uint64_t tot = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
        // pool: every query's partial last chunk plus the results (a guess of 128 per query at first)
        const uint64_t want = attempt == 0 ? std::max<uint64_t>(c.ck_cap, 3 * nq + 1024)
                                           : tot / kResultChunk + nq + 1024;
        if (want > 0xfffffff0ull) return set_error(c, OCT_ERR_INVALID_ARG, "too many results for one call");
        if (want > c.ck_cap) {
            CK(c.ck_pool.reserve(4ull * kResultChunk * want));
            CK(c.ck_next.reserve(4ull * want));
            c.ck_cap = (uint32_t)want;
        }
        ChunkArgs ck{c.ck_pool.as<uint32_t>(), c.ck_next.as<uint32_t>(), c.ck_first.as<uint32_t>(),
                     c.ck_ctr.as<uint32_t>(), c.ck_cap};
        CK(cudaMemsetAsync(ck.ctr, 0, 4, c.stream));
        CK(launch_radius_packet(c, kernel, pass_algo, 2, fp32_on_radius(c.fp32_filter), dq, nq, dr, radius, order,
                                dc, nullptr, nullptr, nullptr, 0, &ck));
        CK(launch_scan_u64(c, dc, doffs, nq));
        CK(cudaMemcpyAsync(c.pinned, doffs + nq, 8, cudaMemcpyDeviceToHost, c.stream));
        const int st = sync_and_check(c, kErrChunkCapacity);
        memcpy(&tot, c.pinned, 8);
        uint32_t* hw = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(c.pinned) + kPinnedErrOffset);
        const bool pool_short = (*hw & kErrChunkCapacity) != 0;
        if (st != OCT_OK) return st;
        if (!pool_short) break;
        if (attempt == 1) return set_error(c, OCT_ERR_DEVICE_LIMIT, "result chunk pool still too small");
    }
    *total = tot;
    return OCT_OK;
}

// One pass into result chunks (radius_chunks), then the chains compacted into the CSR output.
int radius_one_pass(Cloud& c, int kernel, int algo, const double* dq, uint64_t nq, const double* dr, double radius,
                    unsigned long long* doffs, uint64_t* offsets, uint32_t* idx, uint64_t idx_capacity,
                    uint64_t* total, bool dev) {
    uint64_t tot = 0;
    const int st0 = radius_chunks(c, kernel, algo, dq, nq, dr, radius, doffs, &tot);
    if (st0 != OCT_OK) return st0;
    unsigned long long* dc = c.q_counts.as<unsigned long long>();
    if (total) *total = tot;
    if (!dev && offsets) CK(cudaMemcpyAsync(offsets, doffs, 8 * (nq + 1), cudaMemcpyDeviceToHost, c.stream));
    if (tot > idx_capacity || (tot && !idx)) {
        CK(cudaStreamSynchronize(c.stream));
        return set_error(c, OCT_ERR_CAPACITY, "idx capacity smaller than the number of results");
    }
    uint32_t* dout = idx;
    if (!dev) {
        CK(c.q_out.reserve(4 * (tot ? tot : 1)));
        dout = c.q_out.as<uint32_t>();
    }
    ChunkArgs ck{c.ck_pool.as<uint32_t>(), c.ck_next.as<uint32_t>(), c.ck_first.as<uint32_t>(),
                 c.ck_ctr.as<uint32_t>(), c.ck_cap};
    CK(launch_chunk_compact(c.device, c.stream, dc, doffs, ck, dout, tot, nq, nullptr, c.d_err.as<uint32_t>()));
    if (!dev && tot) CK(cudaMemcpyAsync(idx, dout, 4 * tot, cudaMemcpyDeviceToHost, c.stream));
    if (!dev) return sync_and_check(c);
    return OCT_OK;
}

int radius_common(Cloud& c, int kernel, int algo, const double* centers, uint64_t nq, const double* radii,
                  double radius, bool device, const double** dq, const double** dr) {
    if (!c.built) return set_error(c, OCT_ERR_STATE, "search before oct_build");
    if (!valid_kernel(kernel) || !valid_algo(algo)) return set_error(c, OCT_ERR_INVALID_ARG, "bad kernel or algo");
    if (nq && !centers) return set_error(c, OCT_ERR_INVALID_ARG, "centers is NULL");
    int st;
    if ((st = stage_in(c, c.q_centers, centers, 3 * nq, device, dq)) != OCT_OK) return st;
    if ((st = stage_in(c, c.q_radii, radii, nq, device, dr)) != OCT_OK) return st;
    (void)radius;
    return OCT_OK;
}

// Outputs of a finished sort: the Box, keys, permutation, reordered points.
int emit_sorted(Cloud& c, double* box12, uint64_t* keys, uint32_t* perm, double* sorted_xyz, bool dev) {
    int st;
    if (box12) {
        for (int a = 0; a < 3; ++a) {
            box12[a] = c.box.center[a];
            box12[3 + a] = c.box.radii[a];
            box12[6 + a] = c.box.min[a];
            box12[9 + a] = c.box.max[a];
        }
    }
    const uint64_t n = c.n;
    if ((st = copy_out(c, keys, c.keys.as<uint64_t>(), n, dev)) != OCT_OK) return st;
    if ((st = copy_out(c, perm, c.perm.as<uint32_t>(), n, dev)) != OCT_OK) return st;
    if (sorted_xyz && n) {
        double* dst = sorted_xyz;
        if (!dev) {
            CK(c.q_out.reserve(24 * n));
            dst = c.q_out.as<double>();
        }
        k_soa_to_aos<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(c.xs.as<double>(), c.ys.as<double>(),
                                                                        c.zs.as<double>(), n, dst);
        CK(cudaGetLastError());
        if (!dev) CK(cudaMemcpyAsync(sorted_xyz, dst, 24 * n, cudaMemcpyDeviceToHost, c.stream));
    }
    if (!dev) CK(cudaStreamSynchronize(c.stream));
    return OCT_OK;
}

}  // namespace

namespace octb {

cudaMemPool_t cloud_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    if (device < 0 || device >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        // the pool keeps what clouds free, for the next cloud: returning memory to the driver at a
        // synchronisation goes through the driver's resource manager, which a server's other threads
        // would wait on
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[device] = pool;
    }
    return pools[device];
}

static std::mutex g_pinned_mu;
static std::vector<void*> g_pinned_free;

void* pinned_block_get() {
    {
        std::lock_guard<std::mutex> lk(g_pinned_mu);
        if (!g_pinned_free.empty()) {
            void* p = g_pinned_free.back();
            g_pinned_free.pop_back();
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, kPinnedBlock) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void pinned_block_put(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    g_pinned_free.push_back(p);
}

const void* kernel_anchor_capi() { return reinterpret_cast<const void*>(&k_soa_to_aos); }

// The bounded wait of oct_device_wait_probe: poll a flag nothing sets, back off,
// give up after `limit` polls with the error bit set (lane 0 of one warp).
__global__ void k_wait_probe(const uint32_t* flag, uint32_t limit, uint32_t* err, uint32_t* polls) {
    if (threadIdx.x != 0) return;
    uint32_t n = 0;
    for (;;) {
        uint32_t v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
        if (v != 0) break;
        if (++n >= limit) {
            set_err(err, kErrSpinLimit);
            break;
        }
        __nanosleep(64);
    }
    *polls = n;
}

// Every kernel of the library's device code loaded into the current device's
// context: the device library of each source file is found from one of its
// kernels, its kernels enumerated and each loaded (cuFuncLoad, CUDA 12.4+,
// reached through the runtime's driver entry points, so the library does not
// link the driver).  Once per device; a driver without these entry points
// leaves loading to the first launches.
int preload_kernels(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    if (device < 0 || device >= 64) return OCT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(mu);
    if (done[device]) return OCT_OK;
    PFN_cuKernelGetLibrary_v12050 get_lib = nullptr;
    PFN_cuLibraryGetKernelCount_v12040 count_kernels = nullptr;
    PFN_cuLibraryEnumerateKernels_v12040 list_kernels = nullptr;
    PFN_cuKernelGetFunction_v12000 get_func = nullptr;
    PFN_cuFuncLoad_v12040 load = nullptr;
    cudaDriverEntryPointQueryResult q;
    bool ok = cudaGetDriverEntryPointByVersion("cuKernelGetLibrary", reinterpret_cast<void**>(&get_lib), 12050,
                                               cudaEnableDefault, &q) == cudaSuccess && get_lib;
    ok = ok && cudaGetDriverEntryPointByVersion("cuLibraryGetKernelCount", reinterpret_cast<void**>(&count_kernels),
                                                12040, cudaEnableDefault, &q) == cudaSuccess && count_kernels;
    ok = ok && cudaGetDriverEntryPointByVersion("cuLibraryEnumerateKernels", reinterpret_cast<void**>(&list_kernels),
                                                12040, cudaEnableDefault, &q) == cudaSuccess && list_kernels;
    ok = ok && cudaGetDriverEntryPointByVersion("cuKernelGetFunction", reinterpret_cast<void**>(&get_func), 12000,
                                                cudaEnableDefault, &q) == cudaSuccess && get_func;
    ok = ok && cudaGetDriverEntryPointByVersion("cuFuncLoad", reinterpret_cast<void**>(&load), 12040,
                                                cudaEnableDefault, &q) == cudaSuccess && load;
    if (!ok) {
        cudaGetLastError();
        done[device] = true;
        return OCT_OK;
    }
    const void* anchors[] = {kernel_anchor_capi(),          kernel_anchor_encode_sort(),
                             kernel_anchor_engine(),        kernel_anchor_knn_search(),
                             kernel_anchor_octree_build(),  kernel_anchor_radius_packet(),
                             kernel_anchor_radius_search()};
    std::vector<CUkernel> kernels;
    for (const void* a : anchors) {
        cudaKernel_t k = nullptr;
        CUlibrary lib = nullptr;
        unsigned int n = 0;
        if (cudaGetKernel(&k, a) != cudaSuccess || get_lib(&lib, k) != CUDA_SUCCESS ||
            count_kernels(&n, lib) != CUDA_SUCCESS) {
            cudaGetLastError();
            return OCT_ERR_CUDA;
        }
        kernels.resize(n);
        if (n && list_kernels(kernels.data(), n, lib) != CUDA_SUCCESS) return OCT_ERR_CUDA;
        for (CUkernel kk : kernels) {
            CUfunction f = nullptr;
            if (get_func(&f, kk) != CUDA_SUCCESS || load(f) != CUDA_SUCCESS) return OCT_ERR_CUDA;
        }
    }
    done[device] = true;
    return OCT_OK;
}

}  // namespace octb

namespace {
// Every device array of a cloud.
std::vector<DevBuf*> cloud_bufs(Cloud& c) {
    return {&c.xyz_in,   &c.xs,        &c.ys,          &c.zs,          &c.keys,       &c.keys_alt,
            &c.perm,     &c.perm_alt,  &c.keys_hi,     &c.keys_hi_alt, &c.run_pv,     &c.run_pv_alt,
            &c.run_ctl,  &c.run_list,  &c.run_long,  &c.sort_status, &c.d_ctl,       &c.d_box,      &c.d_err,
            &c.offsets,  &c.ranges,    &c.centers,     &c.frontier,    &c.masks,      &c.parts,
            &c.d_build,  &c.q_centers, &c.q_radii,     &c.q_counts,    &c.q_offsets,  &c.q_out,
            &c.q_out2,   &c.q_scan_tmp, &c.qs_keys,    &c.qs_keys_alt, &c.qs_ord,     &c.qs_ord_alt,
            &c.qs_status, &c.qs_ctl,   &c.packet_ctr,  &c.knn_fb,      &c.knn_heads,  &c.stats,
            &c.rel,      &c.crel,      &c.q_axes,      &c.ck_pool,     &c.ck_next,    &c.ck_first,
            &c.ck_ctr};
}
}  // namespace

extern "C" {

int oct_abi_version(void) { return OCT_ABI_VERSION; }

const char* oct_status_string(int s) {
    switch (s) {
        case OCT_OK: return "ok";
        case OCT_ERR_INVALID_ARG: return "invalid argument";
        case OCT_ERR_CUDA: return "CUDA error";
        case OCT_ERR_OUT_OF_MEMORY: return "out of device memory";
        case OCT_ERR_STATE: return "call out of order";
        case OCT_ERR_CAPACITY: return "output capacity too small";
        case OCT_ERR_DEVICE_LIMIT: return "device loop limit reached";
        case OCT_ERR_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

int oct_cloud_create(const oct_params* p, oct_cloud* out) {
    if (!p || !out) return OCT_ERR_INVALID_ARG;
    *out = nullptr;
    if (p->encoder != OCT_ENC_MORTON_3D && p->encoder != OCT_ENC_HILBERT_3D) return OCT_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return OCT_ERR_NO_DEVICE;
    }
    if (p->device < 0 || p->device >= ndev) return OCT_ERR_INVALID_ARG;
    oct_cloud h = new (std::nothrow) oct_cloud_s();
    if (!h) return OCT_ERR_OUT_OF_MEMORY;
    Cloud& c = h->c;
    c.params = *p;
    c.device = p->device;
    c.split_sort = (p->flags & OCT_CLOUD_SORT_8PASS) ? 0 : 1;
    DeviceGuard g(c.device);
    cudaError_t e = cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        c.own_stream = true;
        cudaMemPool_t pool = cloud_pool(c.device);
        if (!pool) e = cudaErrorMemoryAllocation;
        for (DevBuf* b : cloud_bufs(c)) b->bind(pool, &c.stream);
    }
    if (e == cudaSuccess) e = c.d_err.reserve(256);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.d_err.ptr, 0, 256, c.stream);
    if (e == cudaSuccess) e = c.stats.reserve(64);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.stats.ptr, 0, 64, c.stream);
    if (e == cudaSuccess) {
        c.pinned = pinned_block_get();
        if (!c.pinned) e = cudaErrorMemoryAllocation;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        oct_cloud_destroy(h);
        return e == cudaErrorMemoryAllocation ? OCT_ERR_OUT_OF_MEMORY : OCT_ERR_CUDA;
    }
    *out = h;
    return OCT_OK;
}

int oct_cloud_destroy(oct_cloud h) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    {
        DeviceGuard g(c.device);
        if (c.stream) cudaStreamSynchronize(c.stream);
        for (DevBuf* b : cloud_bufs(c)) b->release();  // in the stream's order: waits for nothing else
        if (c.stream) cudaStreamSynchronize(c.stream);
        pinned_block_put(c.pinned);
        for (auto& v : c.ev_pend)
            for (auto& pr : v) c.ev_free.insert(c.ev_free.end(), {pr.first, pr.second});
        for (cudaEvent_t ev : c.ev_free) cudaEventDestroy(ev);
        if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
    }
    delete h;
    return OCT_OK;
}

int oct_cloud_set_stream(oct_cloud h, void* stream) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    CK(cudaStreamSynchronize(c.stream));
    if (c.own_stream) cudaStreamDestroy(c.stream);
    c.own_stream = false;
    c.stream = static_cast<cudaStream_t>(stream);
    return OCT_OK;
}

int oct_last_error(oct_cloud h, char* buf, size_t len) {
    if (!h || !buf || len == 0) return OCT_ERR_INVALID_ARG;
    const std::string& m = h->c.last_error;
    const size_t k = std::min(len - 1, m.size());
    memcpy(buf, m.data(), k);
    buf[k] = '\0';
    return OCT_OK;
}

int oct_synchronize(oct_cloud h) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    return sync_and_check(c);
}

int oct_set_radius_group(oct_cloud h, int lanes) {
    if (!h) return OCT_ERR_INVALID_ARG;
    h->c.radius_group = (lanes == 16 || lanes == 32) ? lanes : 8;
    return OCT_OK;
}

int oct_set_search_config(oct_cloud h, const oct_search_config* cfg) {
    if (!h || !cfg) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    if (cfg->packet < 0 || cfg->packet > 1 || cfg->fp32_filter < 0 || cfg->fp32_filter > OCT_FP32_KNN)
        return set_error(c, OCT_ERR_INVALID_ARG, "packet is 0 or 1, fp32_filter 0-3");
    c.packet = cfg->packet;
    c.fp32_filter = cfg->fp32_filter;
    c.radius_group = (cfg->radius_lanes == 16 || cfg->radius_lanes == 32) ? cfg->radius_lanes : 8;
    c.knn_packet = cfg->knn_packet ? 1 : 0;
    c.knn_bucket = cfg->knn_bucket > 0 ? (uint32_t)cfg->knn_bucket : 0u;
    c.two_pass = cfg->reserved[0] ? 1 : 0;
    // provisional kNN threshold factor in percent: 0 the default, < 0 off
    c.knn_est = cfg->reserved[1] > 0 ? cfg->reserved[1] / 100.0 : (cfg->reserved[1] == 0 ? kKnnEstimate : 0.0);
    if (cfg->reserved[2] < 0 || cfg->reserved[2] > 64)
        return set_error(c, OCT_ERR_INVALID_ARG, "kNN group run length is 0 (default) to 64");
    c.knn_chunk = cfg->reserved[2] > 0 ? (uint32_t)cfg->reserved[2] : kKnnGroupChunk;
    return OCT_OK;
}

int oct_knn_filter_stats(oct_cloud h, uint64_t* point_tests, uint64_t* fp64_tests, uint64_t* band_hits,
                         int reset) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    CK(c.stats.reserve(64));
    unsigned long long v[3] = {0, 0, 0};
    CK(cudaStreamSynchronize(c.stream));
    CK(cudaMemcpy(v, static_cast<unsigned long long*>(c.stats.ptr) + 2, sizeof(v), cudaMemcpyDeviceToHost));
    if (point_tests) *point_tests = v[0];
    if (fp64_tests) *fp64_tests = v[1];
    if (band_hits) *band_hits = v[2];
    if (reset) CK(cudaMemset(static_cast<unsigned long long*>(c.stats.ptr) + 2, 0, sizeof(v)));
    return OCT_OK;
}

int oct_search_stats(oct_cloud h, uint64_t* point_tests, uint64_t* fp64_retests, int reset) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    CK(c.stats.reserve(64));
    unsigned long long v[2] = {0, 0};
    CK(cudaStreamSynchronize(c.stream));
    CK(cudaMemcpy(v, c.stats.ptr, sizeof(v), cudaMemcpyDeviceToHost));
    if (point_tests) *point_tests = v[0];
    if (fp64_retests) *fp64_retests = v[1];
    if (reset) CK(cudaMemset(c.stats.ptr, 0, sizeof(v)));
    return OCT_OK;
}

int oct_cloud_memory(oct_cloud h, uint64_t* bytes) {
    if (!h || !bytes) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    uint64_t s = 0;
    for (const DevBuf* b : cloud_bufs(c)) s += b->bytes;
    *bytes = s;
    return OCT_OK;
}

int oct_device_wait_probe(int device, uint32_t spin_limit, uint32_t* polls) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return OCT_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return OCT_ERR_INVALID_ARG;
    DeviceGuard g(device);
    const uint32_t limit = spin_limit ? spin_limit : kSpinLimit;
    uint32_t* d = nullptr;  // flag, error word, polls
    cudaStream_t s = nullptr;
    uint32_t h[3] = {0, 0, 0};
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&d), 3 * sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d, 0, 3 * sizeof(uint32_t), s);
    if (e == cudaSuccess) {
        k_wait_probe<<<1, 32, 0, s>>>(d, limit, d + 1, d + 2);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (d) cudaFreeAsync(d, s);
    if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return OCT_ERR_CUDA;
    }
    if (polls) *polls = h[2];
    return (h[1] & kErrSpinLimit) ? OCT_ERR_DEVICE_LIMIT : OCT_OK;
}

int oct_trim_cloud_memory(int device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return OCT_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return OCT_ERR_INVALID_ARG;
    cudaMemPool_t pool = cloud_pool(device);
    if (!pool) return OCT_ERR_CUDA;
    DeviceGuard g(device);
    if (cudaMemPoolTrimTo(pool, 0) != cudaSuccess) {
        cudaGetLastError();
        return OCT_ERR_CUDA;
    }
    return OCT_OK;
}

int oct_set_points(oct_cloud h, const double* xyz, uint64_t n, uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    if (n && !xyz) return set_error(c, OCT_ERR_INVALID_ARG, "xyz is NULL");
    if (n >= 0xffffffffull) return set_error(c, OCT_ERR_INVALID_ARG, "more than 2^32 - 2 points");
    DeviceGuard g(c.device);
    CK(c.xyz_in.reserve(24 * (n ? n : 1)));
    if (n) {
        CK(cudaMemcpyAsync(c.xyz_in.ptr, xyz, 24 * n,
                           (flags & OCT_MEM_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.stream));
    }
    c.n = n;
    c.sorted = false;
    c.built = false;
    c.rel_built = false;
    c.crel_built = false;
    c.node_capacity = 0;
    if (!(flags & OCT_MEM_DEVICE)) CK(cudaStreamSynchronize(c.stream));
    return OCT_OK;
}

int oct_encode_sort(oct_cloud h, double* box12, uint64_t* keys, uint32_t* perm, double* sorted_xyz,
                    uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    const bool dev = flags & OCT_MEM_DEVICE;
    if (c.sorted) return emit_sorted(c, box12, keys, perm, sorted_xyz, dev);  // points unchanged since the last sort
    const double* xyz = c.xyz_in.as<double>();
    CK(cudaMemsetAsync(c.d_err.ptr, 0, 4, c.stream));
    const bool split = c.split_sort && c.n;
    CK(launch_bbox_encode(c, xyz, split));
    uint32_t skip[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    auto read_skips = [&]() -> int {  // which digits are the same for every key (their passes are skipped)
        CK(cudaMemcpyAsync(c.pinned, &c.d_ctl.as<SortCtl>()->skip[0], sizeof(skip), cudaMemcpyDeviceToHost,
                           c.stream));
        CK(cudaStreamSynchronize(c.stream));
        memcpy(skip, c.pinned, sizeof(skip));
        return OCT_OK;
    };
    // the split sort (upper halves, then runs; runs longer than 4096 points in a stage of their own).
    // The split sort runs its four passes without reading the skip flags (a pass over a constant digit
    // keeps the order), so nothing waits for the host between the encode and the end of the sort.
    bool done = false;
    unsigned char* pin = static_cast<unsigned char*>(c.pinned);
    if (split) {
        int psel = 0;
        CK(launch_sort_split(c, skip, xyz, &psel));
        // the run flags and the box and level geometry back to the host in one wait
        CK(cudaMemcpyAsync(pin + 2048, c.run_ctl.ptr, 32, cudaMemcpyDeviceToHost, c.stream));
        CK(cudaMemcpyAsync(pin, c.d_box.ptr, sizeof(BoxD) + sizeof(LevelGeom), cudaMemcpyDeviceToHost, c.stream));
        const int st = sync_and_check(c);
        if (st != OCT_OK) return st;
        uint32_t rc[8];  // RunCtl: w_count, w_next, b_count, b_next, big, cap, long-run points, long runs
        memcpy(rc, pin + 2048, sizeof(rc));
        if (rc[4] != 0) {  // runs longer than 4096 points: sorted by their lower halves in a stage of their own
            CK(launch_sort_long(c, xyz, rc[7], rc[6]));
            const int st2 = sync_and_check(c);
            if (st2 != OCT_OK) return st2;
        }
        // the outputs are the sorted cloud
        std::swap(c.keys, c.keys_alt);
        if (psel == 1) std::swap(c.perm, c.perm_alt);
        done = true;
    }
    if (!done) {
        if (c.n) {
            const int st = read_skips();
            if (st != OCT_OK) return st;
        }
        int sel = 0;
        CK(launch_sort_passes(c, skip, &sel));
        if (sel == 1) {
            std::swap(c.keys, c.keys_alt);
            std::swap(c.perm, c.perm_alt);
        }
        CK(launch_gather(c, xyz, c.perm.as<uint32_t>(), 0));
        // box and level geometry back to the host
        CK(cudaMemcpyAsync(pin, c.d_box.ptr, sizeof(BoxD) + sizeof(LevelGeom), cudaMemcpyDeviceToHost, c.stream));
        const int st = sync_and_check(c);
        if (st != OCT_OK) return st;
    }
    memcpy(&c.box, c.pinned, sizeof(BoxD));
    memcpy(&c.geom, static_cast<unsigned char*>(c.pinned) + sizeof(BoxD), sizeof(LevelGeom));
    c.sorted = true;
    c.built = false;
    c.node_capacity = 0;
    return emit_sorted(c, box12, keys, perm, sorted_xyz, dev);
}

int oct_set_sorted_points(oct_cloud h, const double* sorted_xyz, const uint64_t* keys, uint64_t n,
                          const double* box12, uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    if (!box12) return set_error(c, OCT_ERR_INVALID_ARG, "box12 is NULL");
    if (n && (!sorted_xyz || !keys)) return set_error(c, OCT_ERR_INVALID_ARG, "NULL point array");
    if (n >= 0xffffffffull) return set_error(c, OCT_ERR_INVALID_ARG, "more than 2^32 - 2 points");
    const bool dev = flags & OCT_MEM_DEVICE;
    if (!dev) {  // host codes are checked here; device codes are the caller's promise
        for (uint64_t i = 0; i < n; ++i) {
            if (keys[i] >= kUpperBound) return set_error(c, OCT_ERR_INVALID_ARG, "key above 63 bits");
            if (i && keys[i] < keys[i - 1]) return set_error(c, OCT_ERR_INVALID_ARG, "keys are not ascending");
        }
    }
    for (int a = 0; a < 3; ++a)
        if (!(box12[3 + a] >= 0.0)) return set_error(c, OCT_ERR_INVALID_ARG, "negative or NaN box radii");
    DeviceGuard g(c.device);
    const auto kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    CK(c.xyz_in.reserve(24 * (n ? n : 1)));
    CK(c.xs.reserve(8 * (n ? n : 1)));
    CK(c.ys.reserve(8 * (n ? n : 1)));
    CK(c.zs.reserve(8 * (n ? n : 1)));
    CK(c.keys.reserve(8 * (n ? n : 1)));
    CK(c.perm.reserve(4 * (n ? n : 1)));
    CK(c.d_box.reserve(sizeof(BoxD) + sizeof(LevelGeom)));
    // LinearOctree::setupBbox (linear_octree.hpp:439-455) from the caller's Box: half = 0.5f * eps * (max - min),
    // the level radii 2^(21 - l) * half, in the same FP64 operations as the device build
    BoxD box;
    LevelGeom geom;
    const double eps = 4.76837158203125e-07;  // (double)(1.0f / 2^21)
    for (int a = 0; a < 3; ++a) {
        box.center[a] = box12[a];
        box.radii[a] = box12[3 + a];
        box.min[a] = box12[6 + a];
        box.max[a] = box12[9 + a];
        geom.half[a] = (0.5 * eps) * (box.max[a] - box.min[a]);
    }
    for (uint32_t l = 0; l <= kMaxDepth; ++l)
        for (int a = 0; a < 3; ++a) geom.radii[l][a] = (double)(1u << (kMaxDepth - l)) * geom.half[a];
    unsigned char* stage = static_cast<unsigned char*>(c.pinned);
    CK(cudaStreamSynchronize(c.stream));  // the pinned staging area is free
    memcpy(stage, &box, sizeof(BoxD));
    memcpy(stage + sizeof(BoxD), &geom, sizeof(LevelGeom));
    CK(cudaMemcpyAsync(c.d_box.ptr, stage, sizeof(BoxD) + sizeof(LevelGeom), cudaMemcpyHostToDevice, c.stream));
    if (n) {
        CK(cudaMemcpyAsync(c.xyz_in.ptr, sorted_xyz, 24 * n, kind, c.stream));
        CK(cudaMemcpyAsync(c.keys.ptr, keys, 8 * n, kind, c.stream));
        k_aos_to_soa_iota<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(
            c.xyz_in.as<double>(), n, c.xs.as<double>(), c.ys.as<double>(), c.zs.as<double>(), c.perm.as<uint32_t>());
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(c.stream));
    c.n = n;
    c.box = box;
    c.geom = geom;
    c.sorted = true;
    c.built = false;
    c.rel_built = false;
    c.crel_built = false;
    c.node_capacity = 0;
    return OCT_OK;
}

int oct_build(oct_cloud h, oct_tree_info* info) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    if (!c.sorted) return set_error(c, OCT_ERR_STATE, "oct_build before oct_encode_sort");
    DeviceGuard g(c.device);
    for (int attempt = 0; attempt < 8; ++attempt) {
        bool ok = true;
        CK(launch_build(c, &ok));
        CK(cudaMemcpyAsync(c.pinned, c.d_build.ptr, sizeof(BuildCtl), cudaMemcpyDeviceToHost, c.stream));
        const int st = sync_and_check(c, kErrNodeCapacity);
        BuildCtl bc;
        memcpy(&bc, c.pinned, sizeof(BuildCtl));
        if (st != OCT_OK) return st;
        // sync_and_check cleared the word; a capacity miss shows as need_nodes > capacity
        if (bc.need_nodes > c.node_capacity) {
            uint64_t want = std::max<uint64_t>(2ull * bc.need_nodes, 2ull * c.node_capacity);
            if (want > 0xfffffff0ull) want = 0xfffffff0ull;
            if (want <= c.node_capacity) return set_error(c, OCT_ERR_OUT_OF_MEMORY, "octree exceeds 2^32 nodes");
            c.node_capacity = (uint32_t)want;
            continue;
        }
        c.n_total = bc.n_total;
        c.n_internal = bc.n_internal;
        c.n_leaf = bc.n_total - bc.n_internal;
        c.max_depth_seen = bc.max_depth_seen;
        CK(cudaMemsetAsync(c.offsets.as<uint32_t>() + c.n_total, 0, 4, c.stream));
        c.rel_built = false;
        c.crel_built = false;
        if (fp32_on_radius(c.fp32_filter) && c.packet) {  // the FP32 search reads leaf-relative coordinates
            CK(launch_leaf_rel(c));
            c.rel_built = true;
        }
        c.built = true;
        if (info) {
            info->n_points = c.n;
            info->n_leaf = c.n_leaf;
            info->n_internal = c.n_internal;
            info->n_total = c.n_total;
            info->max_depth_seen = c.max_depth_seen;
        }
        return OCT_OK;
    }
    return set_error(c, OCT_ERR_OUT_OF_MEMORY, "octree node capacity retries exhausted");
}

int oct_tree_export(oct_cloud h, uint32_t* offsets, uint64_t* ranges, double* centers, double* radii, double* half,
                    uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    if (!c.built) return set_error(c, OCT_ERR_STATE, "export before oct_build");
    DeviceGuard g(c.device);
    const bool dev = flags & OCT_MEM_DEVICE;
    const uint64_t nt = c.n_total;
    int st;
    if ((st = copy_out(c, offsets, c.offsets.as<uint32_t>(), nt + 1, dev)) != OCT_OK) return st;
    if ((st = copy_out(c, centers, c.centers.as<double>(), 3 * nt, dev)) != OCT_OK) return st;
    if (ranges) {
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(ranges);
        if (!dev) {
            CK(c.q_out2.reserve(16 * nt));
            dst = c.q_out2.as<unsigned long long>();
        }
        k_widen_pairs<<<(unsigned)((nt + 255) / 256), 256, 0, c.stream>>>(c.ranges.as<uint2>(), nt, dst);
        CK(cudaGetLastError());
        if (!dev) CK(cudaMemcpyAsync(ranges, dst, 16 * nt, cudaMemcpyDeviceToHost, c.stream));
    }
    if (radii || half) {
        if (dev) {
            if (radii)
                CK(cudaMemcpyAsync(radii, c.geom.radii, sizeof(c.geom.radii), cudaMemcpyHostToDevice, c.stream));
            if (half) CK(cudaMemcpyAsync(half, c.geom.half, sizeof(c.geom.half), cudaMemcpyHostToDevice, c.stream));
        } else {
            if (radii) memcpy(radii, c.geom.radii, sizeof(c.geom.radii));
            if (half) memcpy(half, c.geom.half, sizeof(c.geom.half));
        }
    }
    CK(cudaStreamSynchronize(c.stream));
    return OCT_OK;
}

int oct_tree_import(oct_cloud h, const oct_tree_info* info, const double* box12, const uint64_t* keys,
                    const uint32_t* perm, const double* sorted_xyz, const uint32_t* offsets, const uint64_t* ranges,
                    const double* centers, const double* radii, const double* half, uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    if (flags != 0) return set_error(c, OCT_ERR_INVALID_ARG, "oct_tree_import takes host buffers (flags 0)");
    if (!info || !box12 || !offsets || !ranges || !centers || !radii || !half)
        return set_error(c, OCT_ERR_INVALID_ARG, "NULL argument");
    const uint64_t n = info->n_points;
    const uint64_t nt = info->n_total;
    if (n >= 0xffffffffull) return set_error(c, OCT_ERR_INVALID_ARG, "more than 2^32 - 2 points");
    if (n && (!keys || !perm || !sorted_xyz)) return set_error(c, OCT_ERR_INVALID_ARG, "NULL point array");
    if (nt == 0 || nt != (uint64_t)info->n_leaf + info->n_internal || nt != 8ull * info->n_internal + 1 ||
        info->max_depth_seen > kMaxDepth)
        return set_error(c, OCT_ERR_INVALID_ARG, "inconsistent tree counts");
    // the checkpoint must describe a valid sorted cloud and tree: nothing is rebuilt
    for (uint64_t i = 1; i < n; ++i)
        if (keys[i] < keys[i - 1]) return set_error(c, OCT_ERR_INVALID_ARG, "keys are not ascending");
    for (uint64_t i = 0; i < n; ++i)
        if (keys[i] >= kUpperBound) return set_error(c, OCT_ERR_INVALID_ARG, "key above 63 bits");
    {
        std::vector<bool> seen(n, false);
        for (uint64_t i = 0; i < n; ++i) {
            if (perm[i] >= n || seen[perm[i]]) return set_error(c, OCT_ERR_INVALID_ARG, "perm is not a permutation");
            seen[perm[i]] = true;
        }
    }
    uint64_t n_parents = 0;
    for (uint64_t i = 0; i < nt; ++i) {
        const uint64_t fc = offsets[i];
        if (fc && (fc <= i || fc + 8 > nt)) return set_error(c, OCT_ERR_INVALID_ARG, "offsets out of range");
        n_parents += fc != 0;
        if (ranges[2 * i] > ranges[2 * i + 1] || ranges[2 * i + 1] > n)
            return set_error(c, OCT_ERR_INVALID_ARG, "ranges out of range");
    }
    if (n_parents != info->n_internal) return set_error(c, OCT_ERR_INVALID_ARG, "offsets do not match n_internal");
    for (uint32_t l = 0; l <= kMaxDepth; ++l)
        for (int a = 0; a < 3; ++a)
            if (!(radii[3 * l + a] >= 0.0)) return set_error(c, OCT_ERR_INVALID_ARG, "negative or NaN radii");
    DeviceGuard g(c.device);
    CK(c.xs.reserve(8 * (n ? n : 1)));
    CK(c.ys.reserve(8 * (n ? n : 1)));
    CK(c.zs.reserve(8 * (n ? n : 1)));
    CK(c.keys.reserve(8 * (n ? n : 1)));
    CK(c.perm.reserve(4 * (n ? n : 1)));
    CK(c.offsets.reserve(4 * (nt + 1)));
    CK(c.ranges.reserve(8 * nt));
    CK(c.centers.reserve(24 * nt));
    CK(c.d_box.reserve(sizeof(BoxD) + sizeof(LevelGeom)));
    CK(c.d_err.reserve(256));
    // host staging: SoA coordinates, 32-bit ranges, the box and level geometry
    std::vector<double> soa(3 * n);
    for (uint64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) soa[a * n + i] = sorted_xyz[3 * i + a];
    std::vector<uint32_t> off32(offsets, offsets + nt);
    off32.push_back(0);  // the sentinel after the last node
    std::vector<uint32_t> rg32(2 * nt);
    for (uint64_t i = 0; i < 2 * nt; ++i) rg32[i] = (uint32_t)ranges[i];
    BoxD box;
    LevelGeom geom;
    for (int a = 0; a < 3; ++a) {
        box.center[a] = box12[a];
        box.radii[a] = box12[3 + a];
        box.min[a] = box12[6 + a];
        box.max[a] = box12[9 + a];
        geom.half[a] = half[a];
    }
    memcpy(geom.radii, radii, sizeof(geom.radii));
    std::vector<unsigned char> bg(sizeof(BoxD) + sizeof(LevelGeom));
    memcpy(bg.data(), &box, sizeof(BoxD));
    memcpy(bg.data() + sizeof(BoxD), &geom, sizeof(LevelGeom));
    const auto H2D = cudaMemcpyHostToDevice;
    if (n) {
        CK(cudaMemcpyAsync(c.xs.ptr, soa.data(), 8 * n, H2D, c.stream));
        CK(cudaMemcpyAsync(c.ys.ptr, soa.data() + n, 8 * n, H2D, c.stream));
        CK(cudaMemcpyAsync(c.zs.ptr, soa.data() + 2 * n, 8 * n, H2D, c.stream));
        CK(cudaMemcpyAsync(c.keys.ptr, keys, 8 * n, H2D, c.stream));
        CK(cudaMemcpyAsync(c.perm.ptr, perm, 4 * n, H2D, c.stream));
    }
    CK(cudaMemcpyAsync(c.offsets.ptr, off32.data(), 4 * (nt + 1), H2D, c.stream));
    CK(cudaMemcpyAsync(c.ranges.ptr, rg32.data(), 8 * nt, H2D, c.stream));
    CK(cudaMemcpyAsync(c.centers.ptr, centers, 24 * nt, H2D, c.stream));
    CK(cudaMemcpyAsync(c.d_box.ptr, bg.data(), bg.size(), H2D, c.stream));
    CK(cudaMemsetAsync(c.d_err.ptr, 0, 4, c.stream));
    CK(cudaStreamSynchronize(c.stream));  // the staging vectors go out of scope
    c.box = box;
    c.geom = geom;
    c.n = n;
    c.n_total = (uint32_t)nt;
    c.n_internal = info->n_internal;
    c.n_leaf = info->n_leaf;
    c.max_depth_seen = info->max_depth_seen;
    c.node_capacity = (uint32_t)nt;
    c.sorted = true;
    c.built = true;
    c.rel_built = false;
    c.crel_built = false;
    if (fp32_on_radius(c.fp32_filter) && c.packet) {  // the FP32 search reads leaf-relative coordinates
        CK(launch_leaf_rel(c));
        c.rel_built = true;
    }
    return sync_and_check(c);
}

int oct_radius_count(oct_cloud h, int kernel, int algo, const double* centers, uint64_t nq, const double* radii,
                     double radius, uint64_t* counts, uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    const bool dev = flags & OCT_MEM_DEVICE;
    const double *dq, *dr;
    int st = radius_common(c, kernel, algo, centers, nq, radii, radius, dev, &dq, &dr);
    if (st != OCT_OK) return st;
    unsigned long long* dc = reinterpret_cast<unsigned long long*>(counts);
    if (!dev || !counts) {
        CK(c.q_counts.reserve(8 * (nq ? nq : 1)));
        dc = c.q_counts.as<unsigned long long>();
    }
    CK(c.q_out2.reserve(8 * (nq ? nq : 1)));
    unsigned long long* dc_ranges = c.q_out2.as<unsigned long long>();
    // for neighborsStruct the reported count is numberOfPoints
    const uint32_t* order = nullptr;
    if (algo == OCT_NEIGHBORS_STRUCT)
        CK(radius_pass(c, kernel, algo, false, dq, nq, dr, radius, dc_ranges, dc, nullptr, nullptr, 0, &order));
    else
        CK(radius_pass(c, kernel, algo, false, dq, nq, dr, radius, dc, nullptr, nullptr, nullptr, 0, &order));
    if (!dev && counts && nq) CK(cudaMemcpyAsync(counts, dc, 8 * nq, cudaMemcpyDeviceToHost, c.stream));
    if (!dev) return sync_and_check(c);
    return OCT_OK;
}

int oct_radius_hash(oct_cloud h, int kernel, int algo, const double* centers, uint64_t nq, const double* radii,
                    double radius, uint64_t* counts, uint64_t* hashes, uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    const bool dev = flags & OCT_MEM_DEVICE;
    if (nq && (!counts || !hashes)) return set_error(c, OCT_ERR_INVALID_ARG, "counts or hashes is NULL");
    const double *dq, *dr;
    int st = radius_common(c, kernel, algo, centers, nq, radii, radius, dev, &dq, &dr);
    if (st != OCT_OK || nq == 0) return st;
    // the one-pass search into result chunks (whatever the cloud's search configuration: the sets are the same),
    // then per query the sum over its chain instead of the CSR lists
    CK(c.q_counts.reserve(8 * nq));
    CK(c.q_offsets.reserve(8 * (nq + 1)));
    uint64_t tot = 0;
    if ((st = radius_chunks(c, kernel, algo, dq, nq, dr, radius, c.q_offsets.as<unsigned long long>(), &tot)) != OCT_OK)
        return st;
    unsigned long long* dh = reinterpret_cast<unsigned long long*>(hashes);
    if (!dev) {
        CK(c.q_out2.reserve(8 * nq));
        dh = c.q_out2.as<unsigned long long>();
    }
    ChunkArgs ck{c.ck_pool.as<uint32_t>(), c.ck_next.as<uint32_t>(), c.ck_first.as<uint32_t>(),
                 c.ck_ctr.as<uint32_t>(), c.ck_cap};
    const unsigned long long* dc = c.q_counts.as<unsigned long long>();
    CK(launch_chunk_hash(c.device, c.stream, dc, ck, dh, nq, c.d_err.as<uint32_t>()));
    if (dev) {
        CK(cudaMemcpyAsync(counts, dc, 8 * nq, cudaMemcpyDeviceToDevice, c.stream));
        return OCT_OK;
    }
    CK(cudaMemcpyAsync(counts, dc, 8 * nq, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(hashes, dh, 8 * nq, cudaMemcpyDeviceToHost, c.stream));
    return sync_and_check(c);
}

int oct_radius_search(oct_cloud h, int kernel, int algo, const double* centers, uint64_t nq, const double* radii,
                      double radius, uint64_t* offsets, uint32_t* idx, uint64_t idx_capacity, uint64_t* total,
                      uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    const bool dev = flags & OCT_MEM_DEVICE;
    const double *dq, *dr;
    int st = radius_common(c, kernel, algo, centers, nq, radii, radius, dev, &dq, &dr);
    if (st != OCT_OK) return st;
    CK(c.q_counts.reserve(8 * (nq ? nq : 1)));
    unsigned long long* dc = c.q_counts.as<unsigned long long>();
    unsigned long long* doffs = reinterpret_cast<unsigned long long*>(offsets);
    if (!dev || !offsets) {
        CK(c.q_offsets.reserve(8 * (nq + 1)));
        doffs = c.q_offsets.as<unsigned long long>();
    }
    const uint32_t* order = nullptr;
    if (c.packet && !c.two_pass && nq)
        return radius_one_pass(c, kernel, algo, dq, nq, dr, radius, doffs, offsets, idx, idx_capacity, total, dev);
    if (algo == OCT_NEIGHBORS_STRUCT) {
        // expanded indices of the ranges: count points, fill as prune-style runs
        CK(c.q_out2.reserve(8 * (nq ? nq : 1)));
        CK(radius_pass(c, kernel, OCT_NEIGHBORS_STRUCT, false, dq, nq, dr, radius, c.q_out2.as<unsigned long long>(),
                       dc, nullptr, nullptr, 0, &order));
    } else {
        CK(radius_pass(c, kernel, algo, false, dq, nq, dr, radius, dc, nullptr, nullptr, nullptr, 0, &order));
    }
    CK(launch_scan_u64(c, dc, doffs, nq));
    CK(cudaMemcpyAsync(c.pinned, doffs + nq, 8, cudaMemcpyDeviceToHost, c.stream));
    if ((st = sync_and_check(c)) != OCT_OK) return st;
    uint64_t tot;
    memcpy(&tot, c.pinned, 8);
    if (total) *total = tot;
    if (!dev && offsets) CK(cudaMemcpyAsync(offsets, doffs, 8 * (nq + 1), cudaMemcpyDeviceToHost, c.stream));
    if (tot > idx_capacity || (tot && !idx)) {
        CK(cudaStreamSynchronize(c.stream));
        return set_error(c, OCT_ERR_CAPACITY, "idx capacity smaller than the number of results");
    }
    uint32_t* dout = idx;
    if (!dev) {
        CK(c.q_out.reserve(4 * (tot ? tot : 1)));
        dout = c.q_out.as<uint32_t>();
    }
    // neighborsStruct's index set equals the points of its ranges; the prune
    // traversal with the same kernel emits exactly that set (same decisions).
    const int fill_algo = (algo == OCT_NEIGHBORS_STRUCT) ? OCT_NEIGHBORS_PRUNE : algo;
    CK(radius_pass(c, kernel, fill_algo, true, dq, nq, dr, radius, nullptr, nullptr, doffs, dout, tot, &order));
    if (!dev && tot) CK(cudaMemcpyAsync(idx, dout, 4 * tot, cudaMemcpyDeviceToHost, c.stream));
    if (!dev) return sync_and_check(c);
    return OCT_OK;
}

namespace {
// The depth cut of a neighborsApprox call, on the cloud for the call's duration.
struct ApproxCut {
    Cloud& c;
    ApproxCut(Cloud& cl, uint32_t cut, int upper) : c(cl) {
        c.approx_cut = cut;
        c.approx_upper = upper;
    }
    ~ApproxCut() {
        c.approx_cut = 0;
        c.approx_upper = 0;
    }
};
}  // namespace

// neighborsStruct, or (approx_cut = precisionLevel + 1) neighborsApprox
static int ranges_search(oct_cloud h, int kernel, const double* centers, uint64_t nq, const double* radii,
                         double radius, uint32_t approx_cut, int approx_upper, uint64_t* range_offsets,
                         uint32_t* pairs, uint64_t pair_capacity, uint64_t* total_ranges, uint64_t* point_counts,
                         uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    ApproxCut cut_scope(c, approx_cut, approx_upper);
    const bool dev = flags & OCT_MEM_DEVICE;
    const double *dq, *dr;
    int st = radius_common(c, kernel, OCT_NEIGHBORS_STRUCT, centers, nq, radii, radius, dev, &dq, &dr);
    if (st != OCT_OK) return st;
    CK(c.q_counts.reserve(8 * (nq ? nq : 1)));
    CK(c.q_out2.reserve(8 * (nq ? nq : 1)));
    unsigned long long* dranges = c.q_counts.as<unsigned long long>();
    unsigned long long* dpoints = reinterpret_cast<unsigned long long*>(point_counts);
    if (!dev || !point_counts) dpoints = c.q_out2.as<unsigned long long>();
    unsigned long long* doffs = reinterpret_cast<unsigned long long*>(range_offsets);
    if (!dev || !range_offsets) {
        CK(c.q_offsets.reserve(8 * (nq + 1)));
        doffs = c.q_offsets.as<unsigned long long>();
    }
    const uint32_t* order = nullptr;
    CK(radius_pass(c, kernel, OCT_NEIGHBORS_STRUCT, false, dq, nq, dr, radius, dranges, dpoints, nullptr, nullptr, 0,
                   &order));
    CK(launch_scan_u64(c, dranges, doffs, nq));
    CK(cudaMemcpyAsync(c.pinned, doffs + nq, 8, cudaMemcpyDeviceToHost, c.stream));
    if ((st = sync_and_check(c)) != OCT_OK) return st;
    uint64_t tot;
    memcpy(&tot, c.pinned, 8);
    if (total_ranges) *total_ranges = tot;
    if (!dev && range_offsets) CK(cudaMemcpyAsync(range_offsets, doffs, 8 * (nq + 1), cudaMemcpyDeviceToHost, c.stream));
    if (!dev && point_counts && nq) CK(cudaMemcpyAsync(point_counts, dpoints, 8 * nq, cudaMemcpyDeviceToHost, c.stream));
    if (tot > pair_capacity || (tot && !pairs)) {
        CK(cudaStreamSynchronize(c.stream));
        return set_error(c, OCT_ERR_CAPACITY, "pair capacity smaller than the number of ranges");
    }
    uint32_t* dout = pairs;
    if (!dev) {
        CK(c.q_out.reserve(8 * (tot ? tot : 1)));
        dout = c.q_out.as<uint32_t>();
    }
    CK(radius_pass(c, kernel, OCT_NEIGHBORS_STRUCT, true, dq, nq, dr, radius, nullptr, nullptr, doffs, dout, tot,
                   &order));
    if (!dev && tot) CK(cudaMemcpyAsync(pairs, dout, 8 * tot, cudaMemcpyDeviceToHost, c.stream));
    if (!dev) return sync_and_check(c);
    return OCT_OK;
}

int oct_struct_search(oct_cloud h, int kernel, const double* centers, uint64_t nq, const double* radii,
                      double radius, uint64_t* range_offsets, uint32_t* pairs, uint64_t pair_capacity,
                      uint64_t* total_ranges, uint64_t* point_counts, uint32_t flags) {
    return ranges_search(h, kernel, centers, nq, radii, radius, 0, 0, range_offsets, pairs, pair_capacity,
                         total_ranges, point_counts, flags);
}

int oct_approx_search(oct_cloud h, int kernel, const double* centers, uint64_t nq, const double* radii,
                      double radius, uint32_t precision_level, int upper_bound, uint64_t* range_offsets,
                      uint32_t* pairs, uint64_t pair_capacity, uint64_t* total_ranges, uint64_t* point_counts,
                      uint32_t flags) {
    // a level at or past the deepest possible node cuts nothing: the neighborsStruct search
    const uint32_t cut = precision_level >= kMaxDepth ? 0u : precision_level + 1;
    return ranges_search(h, kernel, centers, nq, radii, radius, cut, upper_bound ? 1 : 0, range_offsets, pairs,
                         pair_capacity, total_ranges, point_counts, flags);
}

namespace {
// Per-axis radii for the duration of one call.  They are read by the plain
// radius kernel (one group of lanes per query), which the call is routed to.
struct AxesScope {
    Cloud& c;
    int packet;
    AxesScope(Cloud& cl, const double* d_axes, uint32_t stride) : c(cl), packet(cl.packet) {
        c.axes = d_axes;
        c.axes_stride = stride;
        c.packet = 0;
    }
    ~AxesScope() {
        c.axes = nullptr;
        c.axes_stride = 0;
        c.packet = packet;
    }
};

int stage_axes(Cloud& c, int kernel, const double* radii_xyz, uint64_t nq, int per_query, bool dev,
               const double** out) {
    if (kernel != OCT_KERNEL_SQUARE && kernel != OCT_KERNEL_CUBE)
        return set_error(c, OCT_ERR_INVALID_ARG, "per-axis radii take the square or cube kernel");
    if (!radii_xyz && nq) return set_error(c, OCT_ERR_INVALID_ARG, "radii_xyz is NULL");
    if (!radii_xyz) {
        *out = nullptr;
        return OCT_OK;
    }
    return stage_in(c, c.q_axes, radii_xyz, per_query ? 3 * nq : 3, dev, out);
}
}  // namespace

int oct_search_timing(oct_cloud h, int enable) {
    if (!h) return OCT_ERR_INVALID_ARG;
    h->c.time_kernels = enable != 0;
    return OCT_OK;
}

int oct_search_kernel_times(oct_cloud h, double* radius_ms, uint64_t* radius_launches, double* knn_ms,
                            uint64_t* knn_launches, int reset) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    CK(cudaStreamSynchronize(c.stream));
    for (int kind = 0; kind < 2; ++kind) {
        for (auto& pr : c.ev_pend[kind]) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) {
                c.kernel_ms[kind] += ms;
                ++c.kernel_launches[kind];
            }
            cudaGetLastError();
            c.ev_free.push_back(pr.first);
            c.ev_free.push_back(pr.second);
        }
        c.ev_pend[kind].clear();
    }
    if (radius_ms) *radius_ms = c.kernel_ms[0];
    if (radius_launches) *radius_launches = c.kernel_launches[0];
    if (knn_ms) *knn_ms = c.kernel_ms[1];
    if (knn_launches) *knn_launches = c.kernel_launches[1];
    if (reset) {
        c.kernel_ms[0] = c.kernel_ms[1] = 0.0;
        c.kernel_launches[0] = c.kernel_launches[1] = 0;
    }
    return OCT_OK;
}

int oct_radius_search_axes(oct_cloud h, int kernel, int algo, const double* centers, uint64_t nq,
                           const double* radii_xyz, int per_query, uint64_t* offsets, uint32_t* idx,
                           uint64_t idx_capacity, uint64_t* total, uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    const double* da = nullptr;
    const int st = stage_axes(c, kernel, radii_xyz, nq, per_query, (flags & OCT_MEM_DEVICE) != 0, &da);
    if (st != OCT_OK) return st;
    AxesScope scope(c, da, per_query ? 3u : 0u);
    return oct_radius_search(h, kernel, algo, centers, nq, nullptr, 0.0, offsets, idx, idx_capacity, total, flags);
}

int oct_struct_search_axes(oct_cloud h, int kernel, const double* centers, uint64_t nq, const double* radii_xyz,
                           int per_query, uint64_t* range_offsets, uint32_t* pairs, uint64_t pair_capacity,
                           uint64_t* total_ranges, uint64_t* point_counts, uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    DeviceGuard g(c.device);
    const double* da = nullptr;
    const int st = stage_axes(c, kernel, radii_xyz, nq, per_query, (flags & OCT_MEM_DEVICE) != 0, &da);
    if (st != OCT_OK) return st;
    AxesScope scope(c, da, per_query ? 3u : 0u);
    return ranges_search(h, kernel, centers, nq, nullptr, 0.0, 0, 0, range_offsets, pairs, pair_capacity,
                         total_ranges, point_counts, flags);
}

int oct_knn(oct_cloud h, const double* centers, uint64_t nq, uint32_t k, uint32_t* idx, double* d2,
            uint32_t* counts, uint32_t flags) {
    if (!h) return OCT_ERR_INVALID_ARG;
    Cloud& c = h->c;
    if (!c.built) return set_error(c, OCT_ERR_STATE, "knn before oct_build");
    if (k == 0 || k > 1024) return set_error(c, OCT_ERR_INVALID_ARG, "k must be in [1, 1024]");
    if (nq && (!centers || !idx || !d2)) return set_error(c, OCT_ERR_INVALID_ARG, "NULL buffer");
    DeviceGuard g(c.device);
    const bool dev = flags & OCT_MEM_DEVICE;
    const double* dq;
    int st = stage_in(c, c.q_centers, centers, 3 * nq, dev, &dq);
    if (st != OCT_OK) return st;
    uint32_t* di = idx;
    double* dd = d2;
    uint32_t* dc = counts;
    if (!dev) {
        CK(c.q_out.reserve(4 * nq * (uint64_t)k + 4));
        CK(c.q_out2.reserve(8 * nq * (uint64_t)k + 8));
        CK(c.q_counts.reserve(4 * (nq ? nq : 1)));
        di = c.q_out.as<uint32_t>();
        dd = c.q_out2.as<double>();
        dc = counts ? c.q_counts.as<uint32_t>() : nullptr;
    }
    CK(launch_knn(c, dq, nq, k, di, dd, dc));
    if (!dev && nq) {
        CK(cudaMemcpyAsync(idx, di, 4 * nq * (uint64_t)k, cudaMemcpyDeviceToHost, c.stream));
        CK(cudaMemcpyAsync(d2, dd, 8 * nq * (uint64_t)k, cudaMemcpyDeviceToHost, c.stream));
        if (counts) CK(cudaMemcpyAsync(counts, dc, 4 * nq, cudaMemcpyDeviceToHost, c.stream));
    }
    if (!dev) return sync_and_check(c);
    return OCT_OK;
}

}  // extern "C"
