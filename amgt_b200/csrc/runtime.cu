// Library runtime: allocator hooks, per-device state, status strings,
// precision policy, scans and host read-backs.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "amgt_internal.cuh"

namespace amgt {

static std::atomic<uint64_t> g_launches{0};
static thread_local char g_cuda_msg[256];

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line)
{
    snprintf(g_cuda_msg, sizeof(g_cuda_msg), "%s: %s (%s:%d)", cudaGetErrorString(e), what, file, line);
}

// ------------------------------------------------------------- allocator
// Default allocator: a stream-ordered pool owned by the library, one per
// device, that keeps freed memory for reuse (release threshold = max).  The
// device's default pool returns memory to the driver at every synchronize,
// which made each SpGEMM / conversion pay for fresh page mappings.
static cudaMemPool_t g_pools[64];
static std::mutex g_pool_mu;

static cudaMemPool_t library_pool()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    if (g_pools[dev]) return g_pools[dev];
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pools[dev] = pool;
    }
    return g_pools[dev];
}

// Large blocks (>= 32 MiB) are kept when freed and handed to the next
// request of 75-100 % of their size: the pool serves such a request from
// freed memory only by re-mapping it into a new contiguous range, which
// cost 0.3 ms for a 0.5 GB block inside each AMG setup.  A block carries
// an event recorded on the freeing stream; reuse on another stream waits
// for it, and eviction (beyond 8 GiB cached, or amgt_trim_pool) waits for
// it on the host before returning the block to the pool.
struct CachedBlock {
    void *p;
    size_t bytes;
    int dev;
    cudaStream_t stream;
    cudaEvent_t done;
};
static constexpr size_t kCacheMin = 32ull << 20, kCacheCap = 8ull << 30;
static std::mutex g_cache_mu;
static std::vector<CachedBlock> g_cache;                 // freed, kept
static std::unordered_map<void *, size_t> g_big_sizes;  // live large blocks
static size_t g_cache_bytes = 0;

static void release_block(CachedBlock &c)
{
    cudaEventSynchronize(c.done);
    cudaEventDestroy(c.done);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != c.dev) cudaSetDevice(c.dev);
    cudaFreeAsync(c.p, nullptr);  // no use is pending: the event completed
    if (cur != c.dev) cudaSetDevice(cur);
}

// Returns every cached block of `dev` (all devices when dev < 0) to the pool.
static void flush_cache(int dev)
{
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (size_t i = 0; i < g_cache.size();) {
        if (dev < 0 || g_cache[i].dev == dev) {
            g_cache_bytes -= g_cache[i].bytes;
            release_block(g_cache[i]);
            g_cache.erase(g_cache.begin() + (long)i);
        } else {
            ++i;
        }
    }
}

static void *default_alloc(size_t bytes, amgt_stream_t s, void *)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (bytes >= kCacheMin) {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        int best = -1;
        for (int i = 0; i < (int)g_cache.size(); ++i) {
            const CachedBlock &c = g_cache[i];
            if (c.dev == dev && c.bytes >= bytes && bytes >= c.bytes - c.bytes / 4 &&
                (best < 0 || c.bytes < g_cache[best].bytes))
                best = i;
        }
        if (best >= 0) {
            CachedBlock c = g_cache[best];
            g_cache.erase(g_cache.begin() + best);
            g_cache_bytes -= c.bytes;
            if (c.stream != (cudaStream_t)s) cudaStreamWaitEvent((cudaStream_t)s, c.done, 0);
            cudaEventDestroy(c.done);
            g_big_sizes[c.p] = c.bytes;
            return c.p;
        }
    }
    void *p = nullptr;
    cudaMemPool_t pool = library_pool();
    cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, (cudaStream_t)s)
                         : cudaMallocAsync(&p, bytes, (cudaStream_t)s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (bytes >= kCacheMin) {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        g_big_sizes[p] = bytes;
    }
    return p;
}

static void default_free(void *p, amgt_stream_t s, void *)
{
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        auto it = g_big_sizes.find(p);
        if (it != g_big_sizes.end()) {
            CachedBlock c{p, it->second, 0, (cudaStream_t)s, nullptr};
            g_big_sizes.erase(it);
            if (cudaGetDevice(&c.dev) == cudaSuccess &&
                cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming) == cudaSuccess &&
                cudaEventRecord(c.done, (cudaStream_t)s) == cudaSuccess) {
                g_cache.push_back(c);
                g_cache_bytes += c.bytes;
                while (g_cache_bytes > kCacheCap && !g_cache.empty()) {  // oldest first
                    g_cache_bytes -= g_cache.front().bytes;
                    release_block(g_cache.front());
                    g_cache.erase(g_cache.begin());
                }
                return;
            }
            cudaGetLastError();
            if (c.done) cudaEventDestroy(c.done);
        }
    }
    cudaFreeAsync(p, (cudaStream_t)s);
}

// The installed hooks, swapped as one pointer so that a call never pairs
// one installation's function with another's context.  Replaced hook sets
// are kept (a concurrent call may still hold one); each is three words.
struct AllocHooks {
    amgt_alloc_fn alloc;
    amgt_free_fn free;
    void *ctx;
};
static const AllocHooks g_default_hooks{default_alloc, default_free, nullptr};
static std::atomic<const AllocHooks *> g_hooks{&g_default_hooks};
static std::mutex g_hooks_mu;
static std::vector<AllocHooks *> g_hooks_kept;

void *dev_alloc(size_t bytes, cudaStream_t s)
{
    const AllocHooks *h = g_hooks.load(std::memory_order_acquire);
    return h->alloc(bytes, (amgt_stream_t)s, h->ctx);
}
void dev_free(void *p, cudaStream_t s)
{
    const AllocHooks *h = g_hooks.load(std::memory_order_acquire);
    h->free(p, (amgt_stream_t)s, h->ctx);
}

// ---------------------------------------------------------- device state
static constexpr int kMaxDevices = 64;
static DeviceState g_states[kMaxDevices];
static bool g_state_ready[kMaxDevices];
static std::mutex g_state_mu;

int device_state(DeviceState **st)
{
    int dev = 0;
    AMGT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return AMGT_ERR_NO_DEVICE;
    if (g_state_ready[dev]) {
        *st = &g_states[dev];
        return AMGT_OK;
    }
    std::lock_guard<std::mutex> lk(g_state_mu);
    if (!g_state_ready[dev]) {
        DeviceState &s = g_states[dev];
        AMGT_CUDA_TRY(cudaMalloc(&s.err, sizeof(int) * 4));
        AMGT_CUDA_TRY(cudaMemset(s.err, 0, sizeof(int) * 4));
        AMGT_CUDA_TRY(cudaDeviceGetAttribute(&s.sm_count, cudaDevAttrMultiProcessorCount, dev));
        g_state_ready[dev] = true;
    }
    *st = &g_states[dev];
    return AMGT_OK;
}

// The error word as of the last read_back on this device (copied with it
// into pinned slot kErrSlot, so no second synchronisation is needed); a
// raised word is cleared on the stream and reported once.
static constexpr int kErrSlot = 63;

// Pinned staging for read-backs, per host thread and device, so that two
// host threads can read back on one device at once (the AMG setup converts
// its interpolations on a second thread); freed when the thread exits.
struct Staging {
    int64_t *p[kMaxDevices] = {};
    ~Staging()
    {
        for (int64_t *q : p)
            if (q) cudaFreeHost(q);
    }
};
static thread_local Staging g_staging;

static int staging(int64_t **out)
{
    int dev = 0;
    AMGT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return AMGT_ERR_NO_DEVICE;
    if (!g_staging.p[dev]) {
        AMGT_CUDA_TRY(cudaMallocHost(&g_staging.p[dev], sizeof(int64_t) * 64));
        for (int i = 0; i < 64; ++i) g_staging.p[dev][i] = 0;
    }
    *out = g_staging.p[dev];
    return AMGT_OK;
}

// The handles' pinned read-back blocks.  cudaMallocHost can take
// milliseconds in a process that already holds much pinned or device
// memory -- longer than a whole setup's work on the coarse levels -- so
// blocks are kept when a handle is destroyed and handed to the next one of
// a fitting size; they stay until amgt_trim_pool or exit.
static std::mutex g_pin_mu;
static std::multimap<size_t, void *> g_pin_free;       // cached, by size
static std::unordered_map<void *, size_t> g_pin_size;  // every block made here

int pinned_get(size_t bytes, void **out)
{
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_pin_free.lower_bound(bytes);
    if (it != g_pin_free.end() && it->first <= 4 * bytes + 4096) {
        *out = it->second;
        g_pin_free.erase(it);
        return AMGT_OK;
    }
    const size_t sz = (bytes + 4095) & ~(size_t)4095;
    void *p = nullptr;
    AMGT_CUDA_TRY(cudaMallocHost(&p, sz));
    g_pin_size[p] = sz;
    *out = p;
    return AMGT_OK;
}

void pinned_put(void *p)
{
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto s = g_pin_size.find(p);
    if (s == g_pin_size.end()) return;  // not a block of this cache
    g_pin_free.emplace(s->second, p);
}

static void pinned_trim()
{
    std::lock_guard<std::mutex> lk(g_pin_mu);
    for (auto &kv : g_pin_free) {
        g_pin_size.erase(kv.second);
        cudaFreeHost(kv.second);
    }
    g_pin_free.clear();
}

int check_device_error(cudaStream_t s)
{
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    int64_t *pin;
    AMGT_TRY(staging(&pin));
    const int h = (int)pin[kErrSlot];
    if (h != 0) {
        pin[kErrSlot] = 0;
        AMGT_CUDA_TRY(cudaMemsetAsync(st->err, 0, sizeof(int), s));
        snprintf(g_cuda_msg, sizeof(g_cuda_msg), "device error word raised: %d", h);
        return AMGT_ERR_DEVICE;
    }
    return AMGT_OK;
}

int read_back(const int64_t *dev, int count, cudaStream_t s, const int64_t **host)
{
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    if (count > kErrSlot) return AMGT_ERR_INVALID;
    int64_t *pin;
    AMGT_TRY(staging(&pin));
    pin[kErrSlot] = 0;
    AMGT_CUDA_TRY(cudaMemcpyAsync(pin, dev, sizeof(int64_t) * count, cudaMemcpyDeviceToHost, s));
    AMGT_CUDA_TRY(cudaMemcpyAsync(&pin[kErrSlot], st->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    AMGT_CUDA_TRY(cudaStreamSynchronize(s));
    *host = pin;
    return AMGT_OK;
}

// ------------------------------------------------------------------ scans
// Exclusive sum of up to kSmallScan entries in one launch of one CTA
// (CUB's scan takes two launches and a scratch allocation, which dominates
// the small arrays of coarse AMG levels).  Thread t sums a contiguous
// segment, the CTA scans the segment sums, and each thread writes its
// segment; in == out is allowed (every entry is read before it is written).
constexpr int kSmallScan = 32768;

template <typename T>
__global__ void __launch_bounds__(1024) scan_small_kernel(const T *in, T *out, int n)
{
    __shared__ T wsum[32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int per = (n + 1023) / 1024;
    const int b = min(t * per, n), e = min(b + per, n);
    T sum = 0;
    for (int i = b; i < e; ++i) sum += in[i];
    T incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T w = wsum[lane], wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(FULL, wi, o);
            if (lane >= o) wi += y;
        }
        wsum[lane] = wi - w;  // exclusive over warps
    }
    __syncthreads();
    T run = wsum[warp] + incl - sum;
    for (int i = b; i < e; ++i) {
        const T v = in[i];
        out[i] = run;
        run += v;
    }
}

int exclusive_scan_int(const int *in, int *out, int n, cudaStream_t s)
{
    if (n <= 0) return AMGT_OK;
    if (n <= kSmallScan) {
        AMGT_LAUNCH(scan_small_kernel<int>, 1, 1024, 0, s, in, out, n);
        return AMGT_OK;
    }
    size_t bytes = 0;
    AMGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    void *tmp = dev_alloc(bytes ? bytes : 16, s);
    if (!tmp) return AMGT_ERR_ALLOC;
    count_launch();
    cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, s);
    dev_free(tmp, s);
    AMGT_CUDA_TRY(e);
    return AMGT_OK;
}

int exclusive_scan_i64(const int64_t *in, int64_t *out, int n, cudaStream_t s)
{
    if (n <= 0) return AMGT_OK;
    if (n <= kSmallScan) {
        AMGT_LAUNCH(scan_small_kernel<long long>, 1, 1024, 0, s, reinterpret_cast<const long long *>(in),
                    reinterpret_cast<long long *>(out), n);
        return AMGT_OK;
    }
    size_t bytes = 0;
    AMGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    void *tmp = dev_alloc(bytes ? bytes : 16, s);
    if (!tmp) return AMGT_ERR_ALLOC;
    count_launch();
    cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, n, s);
    dev_free(tmp, s);
    AMGT_CUDA_TRY(e);
    return AMGT_OK;
}

// ------------------------------------------------------- precision policy
static int g_policy[32] = {AMGT_DOUBLE, AMGT_FLOAT, AMGT_HALF};
static int g_policy_n = 3;

}  // namespace amgt

using namespace amgt;

extern "C" {

const char *amgt_status_string(int status)
{
    switch (status) {
    case AMGT_OK: return "ok";
    case AMGT_ERR_INVALID: return "invalid argument";
    case AMGT_ERR_ALLOC: return "allocation failed";
    case AMGT_ERR_CUDA: return g_cuda_msg[0] ? g_cuda_msg : "CUDA runtime error";
    case AMGT_ERR_DEVICE: return g_cuda_msg[0] ? g_cuda_msg : "device error word raised";
    case AMGT_ERR_UNSUPPORTED: return "unsupported precision or shape";
    case AMGT_ERR_NO_DEVICE: return "no CUDA device";
    case AMGT_ERR_TOO_LARGE: return "size exceeds the fixed maximum of this entry point";
    default: return "unknown status";
    }
}

int amgt_init(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return AMGT_ERR_NO_DEVICE;
    }
    DeviceState *st;
    return device_state(&st);
}

uint64_t amgt_kernel_launch_count(void) { return g_launches.load(); }

int amgt_kernel_arch(int *binary_version)
{
    if (!binary_version) return AMGT_ERR_INVALID;
    *binary_version = 0;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return AMGT_ERR_NO_DEVICE;
    }
    cudaFuncAttributes fa;
    AMGT_CUDA_TRY(cudaFuncGetAttributes(&fa, scan_small_kernel<int>));
    *binary_version = fa.binaryVersion;
    return AMGT_OK;
}

int amgt_trim_pool(size_t keep_bytes)
{
    cudaMemPool_t pool = library_pool();
    if (!pool) return AMGT_ERR_NO_DEVICE;
    int dev = 0;
    AMGT_CUDA_TRY(cudaGetDevice(&dev));
    flush_cache(dev);
    AMGT_CUDA_TRY(cudaDeviceSynchronize());
    pinned_trim();
    AMGT_CUDA_TRY(cudaMemPoolTrimTo(pool, keep_bytes));
    return AMGT_OK;
}

int amgt_set_allocator(amgt_alloc_fn alloc_fn, amgt_free_fn free_fn, void *ctx)
{
    if ((alloc_fn == nullptr) != (free_fn == nullptr)) return AMGT_ERR_INVALID;
    if (alloc_fn) flush_cache(-1);  // the default allocator's kept blocks go back to its pool
    if (!alloc_fn) {
        g_hooks.store(&g_default_hooks, std::memory_order_release);
        return AMGT_OK;
    }
    std::lock_guard<std::mutex> lk(g_hooks_mu);
    AllocHooks *h = new AllocHooks{alloc_fn, free_fn, ctx};
    g_hooks_kept.push_back(h);
    g_hooks.store(h, std::memory_order_release);
    return AMGT_OK;
}

int amgt_precision_for_level(int level)
{
    if (level < 0) level = 0;
    return g_policy[level < g_policy_n ? level : g_policy_n - 1];
}

int amgt_set_level_policy(const int *prec, int n)
{
    if (n < 0 || n > 32 || (n > 0 && !prec)) return AMGT_ERR_INVALID;
    if (n == 0) {
        g_policy[0] = AMGT_DOUBLE; g_policy[1] = AMGT_FLOAT; g_policy[2] = AMGT_HALF;
        g_policy_n = 3;
        return AMGT_OK;
    }
    for (int i = 0; i < n; ++i)
        if (prec[i] < AMGT_DOUBLE || prec[i] > AMGT_BF16) return AMGT_ERR_INVALID;
    for (int i = 0; i < n; ++i) g_policy[i] = prec[i];
    g_policy_n = n;
    return AMGT_OK;
}

}  // extern "C"
