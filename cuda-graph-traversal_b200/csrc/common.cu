// common.cu -- host helpers shared by every entry point of libg500b.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "g5_common.cuh"

namespace g5 {

static thread_local char t_error[512] = "";

int set_error(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_error, sizeof t_error, fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { t_error[0] = 0; }

int device_info(DeviceInfo *out) {
    static std::mutex mu;
    static DeviceInfo cache[64];
    static bool have[64] = {};
    int dev = 0;
    G5_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64) return set_error(G5_ERR_INVALID, "device ordinal %d out of range", dev);
    if (!have[dev]) {
        DeviceInfo d{dev, 0, 0};
        G5_CUDA_TRY(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
        G5_CUDA_TRY(cudaDeviceGetAttribute(&d.max_threads_per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev));
        cache[dev] = d;
        have[dev] = true;
    }
    *out = cache[dev];
    return G5_OK;
}

int deverr_to_status(unsigned flags, const char *what) {
    if (!flags) return G5_OK;
    if (flags & DEVERR_TIMEOUT)
        return set_error(G5_ERR_TIMEOUT, "%s: a bounded grid barrier wait expired (flags 0x%x)", what, flags);
    if (flags & DEVERR_RANGE)
        return set_error(G5_ERR_INVALID, "%s: input value out of range (flags 0x%x)", what, flags);
    if (flags & DEVERR_DEPTH)
        return set_error(G5_ERR_INVALID, "%s: the graph is deeper than the depth planes hold; raise depth_bits "
                         "(flags 0x%x)", what, flags);
    if (flags & DEVERR_RING)
        return set_error(G5_ERR_INVALID, "%s: an edge weight spans more buckets than the bucket ring holds; "
                         "use a larger delta (flags 0x%x)", what, flags);
    if (flags & DEVERR_DUPLICATE)
        return set_error(G5_ERR_DEVICE, "%s: a bucket or sub-bucket queue held a vertex twice (flags 0x%x)", what,
                         flags);
    if (flags & DEVERR_UNPREPARED)
        return set_error(G5_ERR_INVALID, "%s: workspace not prepared for this graph (flags 0x%x)", what, flags);
    return set_error(G5_ERR_DEVICE, "%s: internal capacity exceeded (flags 0x%x)", what, flags);
}

int l2_persist_window(uint64_t want, uint64_t *bytes) {
    static std::mutex mu;
    static uint64_t reserved[64] = {};
    static int max_window[64] = {}, max_persist[64] = {};
    static bool probed[64] = {};
    *bytes = 0;
    const char *env = getenv("G5_L2_PERSIST");
    if (env && env[0] == '0') return G5_OK;
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    std::lock_guard<std::mutex> lock(mu);
    if (!probed[di.device]) {
        G5_CUDA_TRY(cudaDeviceGetAttribute(&max_window[di.device], cudaDevAttrMaxAccessPolicyWindowSize, di.device));
        G5_CUDA_TRY(cudaDeviceGetAttribute(&max_persist[di.device], cudaDevAttrMaxPersistingL2CacheSize, di.device));
        probed[di.device] = true;
    }
    uint64_t b = std::min<uint64_t>(want, (uint64_t)max_window[di.device]);
    b = std::min<uint64_t>(b, (uint64_t)max_persist[di.device]);
    if (!b) return G5_OK;
    if (reserved[di.device] < b) {
        // Context-level limit: it lasts until this process's context ends.
        G5_CUDA_TRY(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, b));
        reserved[di.device] = b;
    }
    *bytes = b;
    return G5_OK;
}

int persistent_kernel_setup(const void *fn) {
    // G5_SMEM_CARVEOUT (0-100): the preferred shared-memory share of the
    // SM's unified L1/shared array for every persistent search kernel.
    static const int carve = [] {
        const char *s = getenv("G5_SMEM_CARVEOUT");
        return s && *s ? atoi(s) : -1;
    }();
    if (carve >= 0)
        G5_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, carve > 100 ? 100 : carve));
    return G5_OK;
}

unsigned long long wait_limit_ns() {
    static unsigned long long v = [] {
        const char *s = getenv("G5_WAIT_LIMIT_MS");
        unsigned long long ms = s ? strtoull(s, nullptr, 10) : 0;
        if (!ms) ms = 2000;
        return ms * 1000000ull;
    }();
    return v;
}

// Grid barrier whose arrival target is one block more than the grid: it can
// never complete, so every block's bounded wait must expire.
__global__ void selftest_wait_kernel(unsigned *ctl, unsigned long long limit_ns) {
    unsigned epoch = 0;
    grid_sync(&ctl[0], &ctl[1], epoch, gridDim.x + 1, limit_ns);
}

}  // namespace g5

extern "C" int g5_selftest_wait_timeout(unsigned limit_ms, void *d_work, uint64_t work_bytes, void *stream) {
    using namespace g5;
    clear_error();
    G5_CHECK_ARG(d_work && work_bytes >= 2 * sizeof(unsigned), "g5_selftest_wait_timeout: workspace too small");
    G5_CHECK_ARG(limit_ms >= 1 && limit_ms <= 10000, "g5_selftest_wait_timeout: limit outside [1, 10000] ms");
    cudaStream_t st = (cudaStream_t)stream;
    unsigned *ctl = (unsigned *)d_work;
    G5_CUDA_TRY(cudaMemsetAsync(ctl, 0, 2 * sizeof(unsigned), st));
    unsigned long long limit = (unsigned long long)limit_ms * 1000000ull;
    void *args[] = {&ctl, &limit};
    G5_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)selftest_wait_kernel, dim3(2), dim3(32), args, 0, st));
    unsigned flags[2] = {0, 0};
    G5_CUDA_TRY(cudaMemcpyAsync(flags, ctl, sizeof flags, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    return deverr_to_status(flags[1], "g5_selftest_wait_timeout");
}

extern "C" const char *g5_last_error(void) { return g5::t_error; }
extern "C" const char *g5_version(void) { return "g500b 0.1 (sm_100a)"; }
