// dfea_host.cpp -- host side of the C ABI: error reporting, device queries and the greedy element
// colouring that orders the deterministic scatter of every element kernel.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "difffea_b200.h"

namespace dfea {

static thread_local char g_error[512] = "no error";

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
    return code;
}

int check_cuda(cudaError_t err, const char* what) {
    if (err == cudaSuccess) return DFEA_OK;
    return set_error(DFEA_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(err), cudaGetErrorName(err));
}

int launch_check(const char* what) { return check_cuda(cudaGetLastError(), what); }

// Kernels this library has launched in the process (direct launches when issued, graph-executed
// kernels when the graph's solve returns): the evidence behind a benchmark's "gpu_launches".
static std::atomic<long long> g_launches{0};
static thread_local long long t_launches = 0;  // the same count for the calling thread alone
void note_launches(long long n) {
    g_launches.fetch_add(n, std::memory_order_relaxed);
    t_launches += n;
}
long long thread_launch_count() { return t_launches; }

// Page-locked staging for the small reads that end a stream's work (PCG status words, host-driven dot
// products, Lanczos histories).  A device-to-host copy into pageable memory goes through the driver's
// staging path, which all threads of the process share, so with many solver threads waiting on their
// streams the reads queue behind one another.  Blocks are allocated page-locked (portable across
// devices) on first need and reused for the life of the process: the pool holds as many blocks as reads
// were ever in flight at once.  Allocation failure falls back to a pageable read.
static constexpr size_t kHostBlockBytes = 32 * 1024;
static std::mutex g_host_blocks_mutex;
static std::vector<void*> g_host_blocks;

static void* acquire_host_block() {
    {
        std::lock_guard<std::mutex> lock(g_host_blocks_mutex);
        if (!g_host_blocks.empty()) {
            void* p = g_host_blocks.back();
            g_host_blocks.pop_back();
            return p;
        }
    }
    void* p = nullptr;
    if (cudaHostAlloc(&p, kHostBlockBytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

static void release_host_block(void* p) {
    std::lock_guard<std::mutex> lock(g_host_blocks_mutex);
    g_host_blocks.push_back(p);
}

int read_to_host(void* host, const void* dev, size_t bytes, cudaStream_t s) {
    void* block = bytes <= kHostBlockBytes ? acquire_host_block() : nullptr;
    void* dst = block ? block : host;
    int rc = check_cuda(cudaMemcpyAsync(dst, dev, bytes, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync");
    if (!rc) rc = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (block) {
        if (!rc) std::memcpy(host, block, bytes);
        release_host_block(block);
    }
    return rc;
}

int device_sm_count() {
    static std::atomic<int> cache[64];   // 0 until queried; threads that race store the same value
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n == 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

// L2 set-aside for persisting accesses, configured once per device (before any stream capture).
// The tangent product marks the DOF vectors it gathers and scatters as persisting so that the
// streamed moduli do not evict them between colour passes.  A context-level limit: it ends with
// the process.  Returns 0 (no window) where the device or driver does not offer it.
static std::mutex g_l2_mutex;
static long long g_l2_setaside[64];
static long long g_l2_window_max[64];
static bool g_l2_init[64];

long long persisting_l2_bytes(long long* max_window) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    std::lock_guard<std::mutex> lock(g_l2_mutex);
    if (!g_l2_init[dev]) {
        g_l2_init[dev] = true;
        int max_persist = 0, max_win = 0;
        if (cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&max_win, cudaDevAttrMaxAccessPolicyWindowSize, dev) == cudaSuccess &&
            max_persist > 0 && max_win > 0) {
            size_t cur = 0;
            if (cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize) == cudaSuccess && cur < (size_t)max_persist)
                cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, (size_t)max_persist);
            if (cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize) == cudaSuccess) {
                g_l2_setaside[dev] = (long long)cur;
                g_l2_window_max[dev] = max_win;
            }
        }
        cudaGetLastError();  // a refused limit is not an error of the caller
    }
    if (max_window) *max_window = g_l2_window_max[dev];
    return g_l2_setaside[dev];
}

}  // namespace dfea

using namespace dfea;

extern "C" const char* dfea_last_error(void) { return g_error; }

extern "C" int dfea_version(void) { return 10000; }

extern "C" int64_t dfea_launch_count(void) { return (int64_t)g_launches.load(std::memory_order_relaxed); }

// Blocking synchronisation (on != 0) or the default spin/yield heuristic (on == 0) for this process's context
// on `device`: with blocking, a host thread waiting for the GPU sleeps instead of spinning (many serving
// threads on few host cores).
extern "C" int dfea_set_blocking_sync(int32_t device, int32_t on) {
    int rc = check_cuda(cudaSetDevice(device), "cudaSetDevice");
    if (rc) return rc;
    const unsigned int want = on ? cudaDeviceScheduleBlockingSync : cudaDeviceScheduleAuto;
    rc = check_cuda(cudaSetDeviceFlags(want), "cudaSetDeviceFlags");
    if (rc) return rc;
    unsigned int flags = 0;
    rc = check_cuda(cudaGetDeviceFlags(&flags), "cudaGetDeviceFlags");
    if (rc) return rc;
    return (flags & cudaDeviceScheduleMask) == want
               ? DFEA_OK
               : set_error(DFEA_ERR_CUDA, "the scheduling flag was not applied (flags 0x%x)", flags);
}

extern "C" int dfea_element_supported(int32_t nen, int32_t n_q) {
    return (nen == 4 && n_q == 4) || (nen == 9 && n_q == 9) || (nen == 3 && n_q == 1) || (nen == 6 && n_q == 6) ||
           (nen == 8 && n_q == 9);
}

extern "C" int dfea_colour_elements(const int64_t* conn, int64_t n_el, int32_t nen, int64_t n_nodes, int32_t* colour,
                                    int32_t* n_colours) {
    if (n_el < 0 || nen < 1 || n_nodes < 1 || !n_colours || (n_el > 0 && (!conn || !colour)))
        return set_error(DFEA_ERR_INVALID, "dfea_colour_elements: bad arguments");
    // used[node]: bit c set when an element of colour c touches the node
    std::vector<uint64_t> used((size_t)n_nodes, 0ull);
    int32_t n_used = 0;
    for (int64_t e = 0; e < n_el; ++e) {
        uint64_t taken = 0ull;
        for (int a = 0; a < nen; ++a) {
            const int64_t node = conn[e * nen + a];
            if (node < 0 || node >= n_nodes)
                return set_error(DFEA_ERR_INVALID, "element %lld references node %lld outside [0, %lld)", (long long)e,
                                 (long long)node, (long long)n_nodes);
            taken |= used[(size_t)node];
        }
        if (taken == ~0ull) return set_error(DFEA_ERR_COLOURS, "element %lld needs more than %d colours", (long long)e,
                                             DFEA_MAX_COLOURS);
        int c = 0;
        while (taken & (1ull << c)) ++c;
        colour[e] = c;
        if (c + 1 > n_used) n_used = c + 1;
        for (int a = 0; a < nen; ++a) used[(size_t)conn[e * nen + a]] |= (1ull << c);
    }
    *n_colours = n_used > 0 ? n_used : 1;
    return DFEA_OK;
}

// sizeof of the public structs, by name: lets a binding check its mirrors against this build's layout
extern "C" int64_t dfea_struct_size(const char* name) {
    if (!name) return -1;
    struct Entry { const char* name; int64_t size; };
    static const Entry table[] = {
        {"dfea_material", (int64_t)sizeof(dfea_material)},   {"dfea_mesh_view", (int64_t)sizeof(dfea_mesh_view)},
        {"dfea_mg_grid", (int64_t)sizeof(dfea_mg_grid)},     {"dfea_mg_level", (int64_t)sizeof(dfea_mg_level)},
        {"dfea_mg", (int64_t)sizeof(dfea_mg)},               {"dfea_newton", (int64_t)sizeof(dfea_newton)},
        {"dfea_newton_record", (int64_t)sizeof(dfea_newton_record)},
        {"dfea_newton_info", (int64_t)sizeof(dfea_newton_info)},
        {"dfea_rect_spec", (int64_t)sizeof(dfea_rect_spec)},
    };
    for (const Entry& e : table)
        if (std::strcmp(e.name, name) == 0) return e.size;
    return -1;
}
