// ob_shift_noalloc: the shift to the sources with no device allocation at all.
//
// ob_shift takes its block partials, column sums and fold counter from the stream-ordered pool
// on every call. Some callers cannot let a library allocate device memory: a host framework that
// owns and accounts every byte of the device (a serving process with a fixed memory budget, or a
// foreign runtime bound through an FFI that forbids allocations behind its back), or a caller in
// a latency-critical loop that may not risk an allocation's driver call or its implicit
// synchronisation. This variant takes its scratch from a file-scope static device array of a
// fixed, modest size instead, so a call allocates nothing; the caller still passes phi and the
// sources.
//
// Limits and sharing: at most kMaxColumns columns per call (larger requests are rejected with
// OB_ERR_INVALID). Every device that loads this library holds one copy of the array (about
// 129 KiB) until the process exits. Every call on a device shares that copy: the fold counter is
// cleared at the start of each call and every other slot is written before it is read, but two
// calls whose work overlaps on the device (different streams, no ordering between them) race on
// it, so callers must order them. The array's device address is looked up on the first call made
// with a device current, and again whenever that device's context has changed since (a host that
// reset the device gets a new context, in which the old address means nothing); make the first
// call on each device, and the first after a reset, before any stream capture.
#include <cuda.h>

#include <mutex>

#include "ob_internal.cuh"

namespace ob {
namespace {

constexpr int kMaxColumns = 64;
constexpr int kMaxBlocks = 128;
constexpr int kThreads = 256;
// Layout in doubles: partials[kMaxBlocks * kMaxColumns] (double2 each), sums[kMaxColumns]
// (double2 each), then the fold counter (an unsigned int in the last slot).
constexpr int kPartialsOffset = 0;
constexpr int kSumsOffset = 2 * kMaxBlocks * kMaxColumns;
constexpr int kCounterOffset = kSumsOffset + 2 * kMaxColumns;
constexpr int kScratchDoubles = kCounterOffset + 2;

static __device__ __align__(256) double g_shift_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_address_mutex;
// Per device: the scratch's address and the context it was looked up in.
double* g_address[kMaxDevices] = {};
CUcontext g_context[kMaxDevices] = {};

// The driver's cuCtxGetCurrent, reached through the runtime (the library does not link the driver
// library itself, so it still loads on a machine without one).
typedef CUresult (*CtxGetCurrent)(CUcontext*);

CUcontext current_context() {
    static CtxGetCurrent fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []() {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult found = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &found) == cudaSuccess &&
            found == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrent>(p);
        else
            cudaGetLastError();
    });
    CUcontext context = nullptr;
    if (fn == nullptr || fn(&context) != CUDA_SUCCESS) return nullptr;
    return context;
}

// The device address of g_shift_scratch for the current device, looked up when the device has no
// cached address or its current context is not the one the cached address belongs to.
int scratch_address(double** out) {
    int device = 0;
    OB_CUDA(cudaGetDevice(&device));
    OB_REQUIRE(device >= 0 && device < kMaxDevices, "ob_shift_noalloc: device %d out of range",
               device);
    std::lock_guard<std::mutex> lock(g_address_mutex);
    CUcontext context = current_context();
    if (g_address[device] == nullptr || context == nullptr || context != g_context[device]) {
        void* address = nullptr;
        // Also makes the device's primary context current when no runtime call has yet.
        cudaError_t e = cudaGetSymbolAddress(&address, g_shift_scratch);
        if (e != cudaSuccess) return cuda_status(e, "ob_shift_noalloc: cudaGetSymbolAddress");
        context = current_context();
        g_address[device] = static_cast<double*>(address);
        g_context[device] = context;
    }
    *out = g_address[device];
    return OB_OK;
}

// Per column: the sum of phi over its sources and over every vertex (block partials folded in
// block order by the last block), as ob_shift's fold (ordito/kernels/heat.py:3383-3403).
__global__ void noalloc_sums_kernel(const double* __restrict__ phi, int n,
                                    const int* __restrict__ sources,
                                    const int* __restrict__ source_offsets, int n_sources, int k,
                                    double* scratch) {
    __shared__ double reduce[32];
    __shared__ int last;
    double2* partials = reinterpret_cast<double2*>(scratch + kPartialsOffset);
    double2* sums = reinterpret_cast<double2*>(scratch + kSumsOffset);
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + kCounterOffset);
    const int c = blockIdx.y;
    const int s_begin = source_offsets ? source_offsets[c] : 0;
    const int s_end = source_offsets ? source_offsets[c + 1] : n_sources;
    double at_sources = 0.0, everywhere = 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s_end - s_begin; i += stride)
        at_sources += phi[(size_t)sources[s_begin + i] * k + c];
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        everywhere += phi[(size_t)v * k + c];
    const double a = block_sum(at_sources, reduce);
    const double b = block_sum(everywhere, reduce);
    if (threadIdx.x == 0) partials[(size_t)c * gridDim.x + blockIdx.x] = make_double2(a, b);
    if (!last_block_arrived(counter, &last)) return;
    for (int col = threadIdx.x; col < k; col += blockDim.x) {
        double s = 0.0, g = 0.0;
        for (int bx = 0; bx < (int)gridDim.x; ++bx) {
            const double2 p = __ldcg(&partials[(size_t)col * gridDim.x + bx]);
            s += p.x;
            g += p.y;
        }
        sums[col] = make_double2(s, g);
    }
}

// phi -= mean over the sources; flipped when oriented and the mean falls below that offset
// (ordito/kernels/heat.py:3406-3424).
__global__ void noalloc_shift_kernel(double* __restrict__ phi, int n, const double* scratch,
                                     const int* __restrict__ source_offsets, int n_sources, int k,
                                     int orient) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * k) return;
    const double2* sums = reinterpret_cast<const double2*>(scratch + kSumsOffset);
    const int c = (int)(t % k);
    const int count = source_offsets ? source_offsets[c + 1] - source_offsets[c] : n_sources;
    const double2 s = sums[c];
    const double offset = s.x / (double)count;
    const double value = phi[t];
    double shifted = value - offset;
    if (orient != 0 && s.y / (double)n - offset < 0.0) shifted = offset - value;
    phi[t] = shifted;
}

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_shift_noalloc(double* phi, int n_vertices, const int32_t* sources, int n_sources,
                     const int32_t* source_offsets, int n_columns, int orient,
                     ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && n_sources >= 0, "ob_shift_noalloc: negative size");
    OB_REQUIRE(n_columns >= 1 && n_columns <= kMaxColumns,
               "ob_shift_noalloc: n_columns = %d outside [1, %d] (the static scratch's limit)",
               n_columns, kMaxColumns);
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(phi != nullptr && sources != nullptr, "ob_shift_noalloc: null pointer");
    OB_REQUIRE(n_columns == 1 || source_offsets != nullptr,
               "ob_shift_noalloc: several columns need source_offsets");
    OB_REQUIRE(source_offsets != nullptr || n_sources > 0, "ob_shift_noalloc: no sources");
    double* scratch = nullptr;
    int st = scratch_address(&scratch);
    if (st) return st;
    const int blocks = std::max(1, std::min(ceil_div(n_vertices, kThreads * 4), kMaxBlocks));
    // The fold counter must start at zero; everything else is written before it is read.
    OB_CUDA(cudaMemsetAsync(scratch + kCounterOffset, 0, sizeof(unsigned int), stream));
    noalloc_sums_kernel<<<dim3(blocks, n_columns), kThreads, 0, stream>>>(
        phi, n_vertices, sources, source_offsets, n_sources, n_columns, scratch);
    OB_CHECK_LAUNCH("noalloc_sums");
    const long long total = (long long)n_vertices * n_columns;
    noalloc_shift_kernel<<<ceil_div(total, kThreads), kThreads, 0, stream>>>(
        phi, n_vertices, scratch, source_offsets, n_sources, n_columns, orient);
    OB_CHECK_LAUNCH("noalloc_shift");
    return OB_OK;
}

}  // extern "C"
