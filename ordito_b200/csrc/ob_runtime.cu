// Runtime plumbing behind the C ABI: error strings, device memory, copies, streams and events.
#include <atomic>
#include <cstdarg>
#include <cstdio>

#include "ob_internal.cuh"

namespace ob {

static thread_local char g_message[512] = "";
static std::atomic<uint64_t> g_launches{0};

int fail(int status, const char* fmt, ...) {
    va_list args;
    va_start(args, fmt);
    vsnprintf(g_message, sizeof(g_message), fmt, args);
    va_end(args);
    return status;
}

static thread_local int g_suppress = 0;

void count_launch(uint64_t n) {
    if (g_suppress == 0) g_launches.fetch_add(n, std::memory_order_relaxed);
}

void suppress_counting(int delta) { g_suppress += delta; }

int sm_count() {
    static int cached = 0;
    if (cached == 0) {
        int device = 0, count = 0;
        if (cudaGetDevice(&device) == cudaSuccess &&
            cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, device) == cudaSuccess)
            cached = count;
        else
            cached = 148;
    }
    return cached;
}

}  // namespace ob

using namespace ob;

extern "C" {

const char* ob_last_error(void) { return g_message; }

int ob_version(void) { return 1; }

int ob_device_count(int* count) {
    OB_REQUIRE(count != nullptr, "ob_device_count: null output");
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        *count = 0;
        cudaGetLastError();
    }
    return OB_OK;
}

int ob_set_device(int device) {
    OB_CUDA(cudaSetDevice(device));
    return OB_OK;
}

int ob_get_device(int* device) {
    OB_REQUIRE(device != nullptr, "ob_get_device: null output");
    OB_CUDA(cudaGetDevice(device));
    return OB_OK;
}

int ob_malloc(size_t bytes, void** ptr, ob_stream_t stream) {
    OB_REQUIRE(ptr != nullptr, "ob_malloc: null output");
    *ptr = nullptr;
    if (bytes == 0) return OB_OK;
    // Stream-ordered pool allocation: freed blocks return to the device's default pool and are
    // reused without a driver call.
    cudaError_t e = cudaMallocAsync(ptr, bytes, as_stream(stream));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? OB_ERR_NOMEM : OB_ERR_CUDA,
                    "ob_malloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    return OB_OK;
}

int ob_free(void* ptr, ob_stream_t stream) {
    if (ptr == nullptr) return OB_OK;
    OB_CUDA(cudaFreeAsync(ptr, as_stream(stream)));
    return OB_OK;
}

int ob_host_alloc(size_t bytes, void** ptr) {
    OB_REQUIRE(ptr != nullptr, "ob_host_alloc: null output");
    *ptr = nullptr;
    if (bytes == 0) return OB_OK;
    OB_CUDA(cudaMallocHost(ptr, bytes));
    return OB_OK;
}

int ob_host_free(void* ptr) {
    if (ptr == nullptr) return OB_OK;
    OB_CUDA(cudaFreeHost(ptr));
    return OB_OK;
}

int ob_memcpy(void* dst, const void* src, size_t bytes, int kind, ob_stream_t stream, int sync) {
    if (bytes == 0) return OB_OK;
    OB_REQUIRE(dst != nullptr && src != nullptr, "ob_memcpy: null pointer");
    cudaMemcpyKind k;
    switch (kind) {
        case 0: k = cudaMemcpyHostToDevice; break;
        case 1: k = cudaMemcpyDeviceToHost; break;
        case 2: k = cudaMemcpyDeviceToDevice; break;
        case 3: k = cudaMemcpyHostToHost; break;
        default: return fail(OB_ERR_INVALID, "ob_memcpy: unknown kind %d", kind);
    }
    OB_CUDA(cudaMemcpyAsync(dst, src, bytes, k, as_stream(stream)));
    if (sync) OB_CUDA(cudaStreamSynchronize(as_stream(stream)));
    return OB_OK;
}

int ob_memset(void* dst, int value, size_t bytes, ob_stream_t stream) {
    if (bytes == 0) return OB_OK;
    OB_REQUIRE(dst != nullptr, "ob_memset: null pointer");
    OB_CUDA(cudaMemsetAsync(dst, value, bytes, as_stream(stream)));
    return OB_OK;
}

int ob_stream_create(ob_stream_t* stream) {
    OB_REQUIRE(stream != nullptr, "ob_stream_create: null output");
    cudaStream_t s;
    OB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream = reinterpret_cast<ob_stream_t>(s);
    return OB_OK;
}

int ob_stream_destroy(ob_stream_t stream) {
    if (stream == nullptr) return OB_OK;
    OB_CUDA(cudaStreamDestroy(as_stream(stream)));
    return OB_OK;
}

int ob_stream_synchronize(ob_stream_t stream) {
    OB_CUDA(cudaStreamSynchronize(as_stream(stream)));
    return OB_OK;
}

int ob_device_synchronize(void) {
    OB_CUDA(cudaDeviceSynchronize());
    return OB_OK;
}

int ob_event_create(void** event) {
    OB_REQUIRE(event != nullptr, "ob_event_create: null output");
    cudaEvent_t e;
    OB_CUDA(cudaEventCreate(&e));
    *event = reinterpret_cast<void*>(e);
    return OB_OK;
}

int ob_event_destroy(void* event) {
    if (event == nullptr) return OB_OK;
    OB_CUDA(cudaEventDestroy(reinterpret_cast<cudaEvent_t>(event)));
    return OB_OK;
}

int ob_event_record(void* event, ob_stream_t stream) {
    OB_CUDA(cudaEventRecord(reinterpret_cast<cudaEvent_t>(event), as_stream(stream)));
    return OB_OK;
}

int ob_event_elapsed_ms(void* start, void* end, float* ms) {
    OB_REQUIRE(ms != nullptr, "ob_event_elapsed_ms: null output");
    OB_CUDA(cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(end)));
    OB_CUDA(cudaEventElapsedTime(ms, reinterpret_cast<cudaEvent_t>(start),
                                 reinterpret_cast<cudaEvent_t>(end)));
    return OB_OK;
}

int ob_launch_count(uint64_t* count) {
    OB_REQUIRE(count != nullptr, "ob_launch_count: null output");
    *count = g_launches.load(std::memory_order_relaxed);
    return OB_OK;
}

}  // extern "C"
