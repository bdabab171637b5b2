// a1: the "cotmatrix" mesh operator pattern, built deterministically from sorted keys.
//
// Follows ordito/laplacian.py:1212-1299 (directed build), ordito/kernels/laplacian.py:707-748
// (store_operator_keys) and ordito/array.py:1688-1807 (csr_from_keys). Keys are
// row * V + col (uint64); the sort is a stable LSD radix sort over only the bits V * V + 1 needs,
// so equal keys keep the producer's slot order and an entry's contributors (its run of equal sorted
// keys) come out in face order. No value is ever accumulated atomically: the runs are flagged,
// scanned and placed, and each entry's value is formed later from its run.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "ob_internal.cuh"

namespace ob {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ unsigned long long csr_key(int row, int col, int n) {
    const unsigned long long sentinel = (unsigned long long)n * (unsigned long long)n;
    if (row < 0 || row >= n || col < 0 || col >= n) return sentinel;
    return (unsigned long long)row * (unsigned long long)n + (unsigned long long)col;
}

// Tail slots: the sentinel (an unreferenced vertex keeps an empty row) with payload -1.
__global__ void fill_tail(unsigned long long* keys, int* order, long long tail, int n) {
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= n) return;
    keys[tail + v] = (unsigned long long)n * (unsigned long long)n;
    order[tail + v] = -1;
}

// One thread per face: both directions of the edge opposite each corner, payload 3 f + e, and the
// diagonal key of each in-range corner (every face writes the same key into a shared vertex's
// tail slot, so the race is benign).
__global__ void operator_keys(const int* __restrict__ faces, int n_faces, int n,
                              unsigned long long* __restrict__ keys, int* __restrict__ order) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const int c[3] = {faces[3 * f], faces[3 * f + 1], faces[3 * f + 2]};
    const long long base = 6LL * f;
    const long long tail = 6LL * n_faces;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const int i = c[(e + 1) % 3], j = c[(e + 2) % 3];
        keys[base + 2 * e] = csr_key(i, j, n);
        keys[base + 2 * e + 1] = csr_key(j, i, n);
        order[base + 2 * e] = 3 * f + e;
        order[base + 2 * e + 1] = 3 * f + e;
        const int v = c[e];
        if (v >= 0 && v < n) keys[tail + v] = csr_key(v, v, n);
    }
}

__global__ void run_flags(const unsigned long long* __restrict__ keys, long long count,
                          unsigned long long sentinel, int* __restrict__ flags) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const unsigned long long k = keys[i];
    flags[i] = (k < sentinel && (i == 0 || keys[i - 1] != k)) ? 1 : 0;
}

// Places each run as one entry and writes the row bounds (ordito/kernels/array.py:1378-1418,
// csr_row_offsets / csr_out_of_range): a run start that opens a row writes the bound of every row
// from the previous entry's row up to its own, and the last in-range position closes the rest.
__global__ void place_runs(const unsigned long long* __restrict__ keys,
                           const int* __restrict__ inclusive, long long count,
                           unsigned long long sentinel, int n, int* __restrict__ offsets,
                           int* __restrict__ columns, int* __restrict__ run_start) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const unsigned long long key = keys[i];
    if (key >= sentinel) {
        if (i == 0)
            for (int r = 0; r <= n; ++r) offsets[r] = 0;
        return;
    }
    const int row = (int)(key / (unsigned long long)n);
    const int entry = inclusive[i] - 1;
    if (i == 0 || keys[i - 1] != key) {
        columns[entry] = (int)(key % (unsigned long long)n);
        run_start[entry] = (int)i;
        const int previous = (i == 0) ? -1 : (int)(keys[i - 1] / (unsigned long long)n);
        for (int r = previous + 1; r <= row; ++r) offsets[r] = entry;
    }
    if (i + 1 == count || keys[i + 1] >= sentinel)
        for (int r = row + 1; r <= n; ++r) offsets[r] = inclusive[i];
}

int key_bits(unsigned long long value) {
    // Bits needed to order keys below `value` (value >= 1).
    int bits = 0;
    unsigned long long v = value - 1;
    while (v) {
        ++bits;
        v >>= 1;
    }
    return bits < 1 ? 1 : bits;
}

struct PatternLayout {
    size_t keys_in = 0, order_in = 0, flags = 0, sort_temp = 0, scan_temp = 0, total = 0;
};

int pattern_layout(int n, int n_faces, PatternLayout* out) {
    const long long count = 6LL * n_faces + n;
    PatternLayout l;
    size_t sort_bytes = 0, scan_bytes = 0;
    if (count > 0) {
        const int end_bit = key_bits((unsigned long long)n * (unsigned long long)n + 1ULL);
        OB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes,
                                                (const unsigned long long*)nullptr,
                                                (unsigned long long*)nullptr, (const int*)nullptr,
                                                (int*)nullptr, (int)count, 0, end_bit));
        OB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, (const int*)nullptr,
                                              (int*)nullptr, (int)count));
    }
    l.keys_in = 0;
    l.order_in = align_up(l.keys_in + 8 * (size_t)count);
    l.flags = align_up(l.order_in + 4 * (size_t)count);
    l.sort_temp = align_up(l.flags + 4 * (size_t)count);
    l.scan_temp = align_up(l.sort_temp + sort_bytes);
    l.total = align_up(l.scan_temp + scan_bytes) + 256;
    *out = l;
    return OB_OK;
}

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_pattern_workspace(int n_vertices, int n_faces, size_t* bytes) {
    OB_REQUIRE(bytes != nullptr, "ob_pattern_workspace: null output");
    OB_REQUIRE(n_vertices >= 0 && n_faces >= 0, "ob_pattern_workspace: negative size");
    OB_REQUIRE(6LL * n_faces + n_vertices < (1LL << 31),
               "ob_pattern_workspace: 6 F + V = %lld keys exceed int32 indexing",
               6LL * n_faces + n_vertices);
    OB_REQUIRE((long long)n_vertices * n_vertices < (1LL << 62), "ob_pattern_workspace: V too large");
    PatternLayout l;
    int st = pattern_layout(n_vertices, n_faces, &l);
    if (st) return st;
    *bytes = l.total;
    return OB_OK;
}

int ob_pattern_build(const int32_t* faces, int n_faces, int n_vertices, int32_t* offsets,
                     int32_t* columns, int32_t* run_start, uint64_t* keys, int32_t* order,
                     void* workspace, size_t workspace_bytes, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && n_faces >= 0, "ob_pattern_build: negative size");
    OB_REQUIRE(offsets != nullptr, "ob_pattern_build: null offsets");
    const long long count = 6LL * n_faces + n_vertices;
    PatternLayout l;
    int st = pattern_layout(n_vertices, n_faces, &l);
    if (st) return st;
    if (count == 0) {
        OB_CUDA(cudaMemsetAsync(offsets, 0, sizeof(int) * (size_t)(n_vertices + 1), stream));
        return OB_OK;
    }
    OB_REQUIRE(faces != nullptr || n_faces == 0, "ob_pattern_build: null faces");
    OB_REQUIRE(columns && run_start && keys && order, "ob_pattern_build: null output");
    OB_REQUIRE(workspace != nullptr && workspace_bytes >= l.total,
               "ob_pattern_build: workspace of %zu bytes, %zu needed", workspace_bytes, l.total);
    char* ws = reinterpret_cast<char*>(align_up(reinterpret_cast<size_t>(workspace)));
    auto* keys_in = reinterpret_cast<unsigned long long*>(ws + l.keys_in);
    auto* order_in = reinterpret_cast<int*>(ws + l.order_in);
    auto* flags = reinterpret_cast<int*>(ws + l.flags);
    void* sort_temp = ws + l.sort_temp;
    void* scan_temp = ws + l.scan_temp;
    const long long tail = 6LL * n_faces;
    if (n_vertices > 0) {
        fill_tail<<<ceil_div(n_vertices, kThreads), kThreads, 0, stream>>>(keys_in, order_in, tail,
                                                                           n_vertices);
        OB_CHECK_LAUNCH("fill_tail");
    }
    if (n_faces > 0) {
        operator_keys<<<ceil_div(n_faces, kThreads), kThreads, 0, stream>>>(faces, n_faces,
                                                                            n_vertices, keys_in,
                                                                            order_in);
        OB_CHECK_LAUNCH("operator_keys");
    }
    const unsigned long long sentinel = (unsigned long long)n_vertices * n_vertices;
    const int end_bit = key_bits(sentinel + 1ULL);
    size_t sort_bytes = l.scan_temp - l.sort_temp;
    OB_CUDA(cub::DeviceRadixSort::SortPairs(sort_temp, sort_bytes, keys_in,
                                            reinterpret_cast<unsigned long long*>(keys), order_in,
                                            order, (int)count, 0, end_bit, stream));
    count_launch(1);
    const int blocks = ceil_div(count, kThreads);
    run_flags<<<blocks, kThreads, 0, stream>>>(reinterpret_cast<unsigned long long*>(keys), count,
                                               sentinel, flags);
    OB_CHECK_LAUNCH("run_flags");
    size_t scan_bytes = l.total - 256 - l.scan_temp;
    OB_CUDA(cub::DeviceScan::InclusiveSum(scan_temp, scan_bytes, flags, flags, (int)count, stream));
    count_launch(1);
    place_runs<<<blocks, kThreads, 0, stream>>>(reinterpret_cast<unsigned long long*>(keys), flags,
                                                count, sentinel, n_vertices, offsets, columns,
                                                run_start);
    OB_CHECK_LAUNCH("place_runs");
    return OB_OK;
}

}  // extern "C"
