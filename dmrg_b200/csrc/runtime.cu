#include <atomic>
// Library runtime: thread-local error text, device queries and the per-(device, stream)
// scratch workspaces used by the stateless entry points (heff_matvec_*, heff_expval_*, ...).
#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <utility>

#include "runtime.cuh"

namespace heff {

static thread_local char g_last_error[512] = "";

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
    snprintf(g_last_error, sizeof(g_last_error), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
}

void set_last_error_msg(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

static std::atomic<int64_t> g_matvec_launches{0};
void count_launches(int64_t n) { g_matvec_launches.fetch_add(n, std::memory_order_relaxed); }

int device_sm_count() {
    static int cache[64] = {0};
    int        dev       = 0;
    if(cudaGetDevice(&dev) != cudaSuccess) return 148;
    if(dev >= 0 && dev < 64 && cache[dev]) return cache[dev];
    int n = 0;
    if(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    if(dev >= 0 && dev < 64) cache[dev] = n;
    return n;
}

struct WsKey {
    int          dev;
    cudaStream_t stream;
    bool         operator<(const WsKey &o) const { return dev != o.dev ? dev < o.dev : (uintptr_t)stream < (uintptr_t)o.stream; }
};
struct WsBuf {
    void  *ptr   = nullptr;
    size_t bytes = 0;
};
static std::mutex              g_ws_mutex;
static std::map<WsKey, WsBuf> *g_ws = nullptr;

int stream_workspace(cudaStream_t stream, size_t bytes, void **out) {
    int dev = 0;
    HEFF_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    if(!g_ws) g_ws = new std::map<WsKey, WsBuf>();
    WsBuf &b = (*g_ws)[WsKey{dev, stream}];
    if(b.bytes < bytes) {
        // Growth reallocates: wait for work that may still read the old buffer on this stream.
        if(b.ptr) {
            HEFF_CUDA(cudaStreamSynchronize(stream));
            HEFF_CUDA(cudaFree(b.ptr));
            b.ptr   = nullptr;
            b.bytes = 0;
        }
        size_t want = bytes + bytes / 4 + 256;
        HEFF_CUDA(cudaMalloc(&b.ptr, want));
        b.bytes = want;
    }
    *out = b.ptr;
    return HEFF_OK;
}

int release_workspaces() {
    std::lock_guard<std::mutex> lock(g_ws_mutex);
    if(!g_ws) return HEFF_OK;
    int cur = 0;
    cudaGetDevice(&cur);
    for(auto &kv : *g_ws) {
        if(kv.second.ptr) {
            cudaSetDevice(kv.first.dev);
            cudaStreamSynchronize(kv.first.stream);
            cudaFree(kv.second.ptr);
        }
    }
    g_ws->clear();
    cudaSetDevice(cur);
    return HEFF_OK;
}

}  // namespace heff

extern "C" const char *heff_last_error(void) { return heff::g_last_error; }
extern "C" const char *heff_version(void) { return "heff_b200 0.1 (sm_100a)"; }

extern "C" int64_t heff_matvec_launches(void) { return heff::g_matvec_launches.load(); }
