// Runtime plumbing behind the C ABI: error strings, device memory, copies, streams and events.
#include <atomic>
#include <vector>
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

std::recursive_mutex& capture_mutex() {
    static std::recursive_mutex mutex;
    return mutex;
}

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

namespace {

constexpr int kMaxDevices = 64;
std::atomic<int> g_pool_kept[kMaxDevices];

// The current device's default pool, set (once per device) to keep freed memory.
cudaError_t kept_pool(cudaMemPool_t* pool) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetDefaultMemPool(pool, device);
    if (e != cudaSuccess) return e;
    if (device >= 0 && device < kMaxDevices &&
        g_pool_kept[device].load(std::memory_order_acquire) == 0) {
        uint64_t keep = ~uint64_t(0);
        e = cudaMemPoolSetAttribute(*pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
        g_pool_kept[device].store(1, std::memory_order_release);
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t pool_malloc(void** p, size_t bytes, cudaStream_t stream) {
    cudaMemPool_t pool;
    const cudaError_t e = kept_pool(&pool);
    if (e != cudaSuccess) return e;
    return cudaMallocAsync(p, bytes, stream);
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
    cudaError_t e = pool_malloc(ptr, bytes, as_stream(stream));
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
    std::lock_guard<std::recursive_mutex> guard(capture_mutex());
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

int ob_event_synchronize(void* event) {
    OB_REQUIRE(event != nullptr, "ob_event_synchronize: null event");
    OB_CUDA(cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(event)));
    return OB_OK;
}

int ob_stream_wait_event(ob_stream_t stream, void* event) {
    OB_REQUIRE(event != nullptr, "ob_stream_wait_event: null event");
    OB_CUDA(cudaStreamWaitEvent(as_stream(stream), reinterpret_cast<cudaEvent_t>(event), 0));
    return OB_OK;
}

int ob_event_query(void* event, int* done) {
    OB_REQUIRE(event != nullptr && done != nullptr, "ob_event_query: bad argument");
    const cudaError_t e = cudaEventQuery(reinterpret_cast<cudaEvent_t>(event));
    if (e == cudaErrorNotReady) {
        cudaGetLastError();  // not an error: clear it
        *done = 0;
        return OB_OK;
    }
    OB_CUDA(e);
    *done = 1;
    return OB_OK;
}

int ob_mem_info(size_t* free_bytes, size_t* total_bytes) {
    OB_REQUIRE(free_bytes != nullptr && total_bytes != nullptr, "ob_mem_info: bad argument");
    OB_CUDA(cudaMemGetInfo(free_bytes, total_bytes));
    // Memory the library's pool keeps but no allocation uses is free to the library.
    cudaMemPool_t pool;
    OB_CUDA(kept_pool(&pool));
    uint64_t reserved = 0, used = 0;
    OB_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    OB_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
    if (reserved > used) *free_bytes += static_cast<size_t>(reserved - used);
    return OB_OK;
}

int ob_mem_trim(size_t keep_bytes) {
    cudaMemPool_t pool;
    OB_CUDA(kept_pool(&pool));
    OB_CUDA(cudaDeviceSynchronize());
    OB_CUDA(cudaMemPoolTrimTo(pool, keep_bytes));
    return OB_OK;
}

namespace {

// A recorded graph and the kernel launches one replay makes (child graphs included).
struct RecordedGraph {
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
};

int count_kernels(cudaGraph_t graph, int depth = 0) {
    size_t count = 0;
    if (depth > 8 || cudaGraphGetNodes(graph, nullptr, &count) != cudaSuccess || count == 0) return 0;
    std::vector<cudaGraphNode_t> nodes(count);
    if (cudaGraphGetNodes(graph, nodes.data(), &count) != cudaSuccess) return 0;
    int kernels = 0;
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType type;
        if (cudaGraphNodeGetType(node, &type) != cudaSuccess) continue;
        if (type == cudaGraphNodeTypeKernel) {
            ++kernels;
        } else if (type == cudaGraphNodeTypeGraph) {
            cudaGraph_t child = nullptr;
            if (cudaGraphChildGraphNodeGetGraph(node, &child) == cudaSuccess) kernels += count_kernels(child, depth + 1);
        }
    }
    return kernels;
}

}  // namespace

int ob_capture_begin(ob_stream_t stream) {
    OB_REQUIRE(stream != nullptr, "ob_capture_begin: capture needs a created stream, not the default");
    capture_mutex().lock();  // held until ob_capture_end on this thread
    const cudaError_t e = cudaStreamBeginCapture(as_stream(stream), cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        capture_mutex().unlock();
        return cuda_status(e, "ob_capture_begin");
    }
    suppress_counting(1);
    return OB_OK;
}

int ob_capture_end(ob_stream_t stream, void** graph, int* kernels) {
    OB_REQUIRE(stream != nullptr && graph != nullptr, "ob_capture_end: bad argument");
    *graph = nullptr;
    suppress_counting(-1);
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture(as_stream(stream), &captured);
    capture_mutex().unlock();
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (captured) cudaGraphDestroy(captured);
        return cuda_status(e, "ob_capture_end");
    }
    auto* recorded = new RecordedGraph;
    recorded->kernels = count_kernels(captured);
    e = cudaGraphInstantiate(&recorded->exec, captured, 0);
    cudaGraphDestroy(captured);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete recorded;
        return cuda_status(e, "ob_capture_end: instantiate");
    }
    if (kernels) *kernels = recorded->kernels;
    *graph = recorded;
    return OB_OK;
}

int ob_graph_launch(void* graph, ob_stream_t stream) {
    OB_REQUIRE(graph != nullptr, "ob_graph_launch: null graph");
    auto* recorded = static_cast<RecordedGraph*>(graph);
    OB_CUDA(cudaGraphLaunch(recorded->exec, as_stream(stream)));
    count_launch((uint64_t)recorded->kernels);
    return OB_OK;
}

int ob_graph_destroy(void* graph) {
    if (graph == nullptr) return OB_OK;
    auto* recorded = static_cast<RecordedGraph*>(graph);
    cudaGraphExecDestroy(recorded->exec);
    delete recorded;
    return OB_OK;
}

int ob_launch_count(uint64_t* count) {
    OB_REQUIRE(count != nullptr, "ob_launch_count: null output");
    *count = g_launches.load(std::memory_order_relaxed);
    return OB_OK;
}

}  // extern "C"
