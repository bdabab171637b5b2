// Shared internals of libordito_b200: status plumbing, launch accounting and block reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/ordito_b200.h"

namespace ob {

// Records a one-line error message for ob_last_error() and returns the status.
int fail(int status, const char* fmt, ...);

// Counts this library's kernel launches (ob_launch_count). While a graph is being captured the
// count is suppressed (suppress_counting(+1) ... (-1)); its replays are counted by the caller.
void count_launch(uint64_t n = 1);
void suppress_counting(int delta);

inline int cuda_status(cudaError_t err, const char* what) {
    if (err == cudaSuccess) return OB_OK;
    if (err == cudaErrorMemoryAllocation) return fail(OB_ERR_NOMEM, "%s: %s", what, cudaGetErrorString(err));
    return fail(OB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(err));
}

#define OB_CUDA(call)                                                      \
    do {                                                                   \
        cudaError_t _e = (call);                                           \
        if (_e != cudaSuccess) return ::ob::cuda_status(_e, #call);        \
    } while (0)

#define OB_CHECK_LAUNCH(name)                                              \
    do {                                                                   \
        ::ob::count_launch();                                              \
        cudaError_t _e = cudaGetLastError();                               \
        if (_e != cudaSuccess) return ::ob::cuda_status(_e, name);         \
    } while (0)

#define OB_REQUIRE(cond, ...)                                              \
    do {                                                                   \
        if (!(cond)) return ::ob::fail(OB_ERR_INVALID, __VA_ARGS__);       \
    } while (0)

inline cudaStream_t as_stream(ob_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

inline int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

inline size_t align_up(size_t bytes, size_t alignment = 256) {
    return (bytes + alignment - 1) / alignment * alignment;
}

// Serialises graph captures against device-wide synchronisation across host threads: a
// cudaDeviceSynchronize while any thread's stream is capturing fails (and invalidates nothing
// only because it is refused). Every capture holds it from begin to end, every device-wide
// synchronisation while it runs; recursive, so a capturing thread may take it again.
std::recursive_mutex& capture_mutex();

// Number of SMs of the current device (cached per process; the library targets one device model).
int sm_count();

// Every device allocation of the library: stream-ordered, from the current device's default
// memory pool. The first call on a device sets that pool to keep the memory freed into it across
// synchronisations (the pool's default hands it back to the driver at every synchronise, and the
// next call's allocations then map fresh pages: tens of milliseconds, varying from call to call,
// for a call that allocates and frees its scratch each time). ob_mem_trim releases it.
cudaError_t pool_malloc(void** p, size_t bytes, cudaStream_t stream);

// Warp-level sum.
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum in a fixed tree (bit-reproducible for a fixed launch shape). Every thread gets
// the result. `scratch` holds blockDim.x / 32 values.
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    T total = (lane < nw) ? scratch[lane] : T(0);
    total = warp_sum(total);
    return total;
}

template <typename T>
__device__ __forceinline__ T block_max(T v, T* scratch, T lowest) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    T total = (lane < nw) ? scratch[lane] : lowest;
    return warp_max(total);
}

// "Last block folds" ticket: returns true in every thread of the block that arrives last at
// `counter` (which it then resets to 0 for the next launch). The block must have published its
// partial (by thread 0) before calling; the fence orders that write before the ticket.
__device__ __forceinline__ bool last_block_arrived(unsigned int* counter, int* shared_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int ticket = atomicAdd(counter, 1u);
        const unsigned int blocks = gridDim.x * gridDim.y * gridDim.z;
        *shared_flag = (ticket == blocks - 1);
        if (ticket == blocks - 1) {
            *counter = 0u;
            __threadfence();
        }
    }
    __syncthreads();
    return *shared_flag != 0;
}

}  // namespace ob
