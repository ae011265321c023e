// Library runtime: allocator hooks, per-device state, status strings,
// precision policy, scans and host read-backs.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>

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

static void *default_alloc(size_t bytes, amgt_stream_t s, void *)
{
    void *p = nullptr;
    cudaMemPool_t pool = library_pool();
    cudaError_t e = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, (cudaStream_t)s)
                         : cudaMallocAsync(&p, bytes, (cudaStream_t)s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

static void default_free(void *p, amgt_stream_t s, void *)
{
    cudaFreeAsync(p, (cudaStream_t)s);
}

static amgt_alloc_fn g_alloc = default_alloc;
static amgt_free_fn g_free = default_free;
static void *g_alloc_ctx = nullptr;

void *dev_alloc(size_t bytes, cudaStream_t s) { return g_alloc(bytes, (amgt_stream_t)s, g_alloc_ctx); }
void dev_free(void *p, cudaStream_t s) { g_free(p, (amgt_stream_t)s, g_alloc_ctx); }

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
        AMGT_CUDA_TRY(cudaMallocHost(&s.pinned, sizeof(int64_t) * 16));
        AMGT_CUDA_TRY(cudaDeviceGetAttribute(&s.sm_count, cudaDevAttrMultiProcessorCount, dev));
        g_state_ready[dev] = true;
    }
    *st = &g_states[dev];
    return AMGT_OK;
}

int check_device_error(cudaStream_t s)
{
    DeviceState *st;
    AMGT_TRY(device_state(&st));
    int h = 0;
    AMGT_CUDA_TRY(cudaMemcpyAsync(&h, st->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    AMGT_CUDA_TRY(cudaStreamSynchronize(s));
    if (h != 0) {
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
    AMGT_CUDA_TRY(cudaMemcpyAsync(st->pinned, dev, sizeof(int64_t) * count, cudaMemcpyDeviceToHost, s));
    AMGT_CUDA_TRY(cudaStreamSynchronize(s));
    *host = st->pinned;
    return AMGT_OK;
}

// ------------------------------------------------------------------ scans
int exclusive_scan_int(const int *in, int *out, int n, cudaStream_t s)
{
    if (n <= 0) return AMGT_OK;
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

int amgt_trim_pool(size_t keep_bytes)
{
    cudaMemPool_t pool = library_pool();
    if (!pool) return AMGT_ERR_NO_DEVICE;
    AMGT_CUDA_TRY(cudaDeviceSynchronize());
    AMGT_CUDA_TRY(cudaMemPoolTrimTo(pool, keep_bytes));
    return AMGT_OK;
}

int amgt_set_allocator(amgt_alloc_fn alloc_fn, amgt_free_fn free_fn, void *ctx)
{
    if ((alloc_fn == nullptr) != (free_fn == nullptr)) return AMGT_ERR_INVALID;
    g_alloc = alloc_fn ? alloc_fn : default_alloc;
    g_free = free_fn ? free_fn : default_free;
    g_alloc_ctx = alloc_fn ? ctx : nullptr;
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
