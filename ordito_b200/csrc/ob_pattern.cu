// a1: the "cotmatrix" mesh operator pattern, built deterministically from sorted keys.
//
// Follows ordito/laplacian.py:1212-1299 (directed build), ordito/kernels/laplacian.py:707-748
// (store_operator_keys) and ordito/array.py:1688-1807 (csr_from_keys). Keys are
// row * V + col (uint64), sorted stably: equal keys keep the producer's slot order, so an entry's
// contributors (its run of equal sorted keys) come out in face order. The sort is by row buckets:
// each in-range key counted into its row and scattered into the row's bucket as (col, slot), each
// bucket sorted by (col, slot) -- the order a stable sort by key gives, whatever order the scatter
// filled the bucket in -- and the out-of-range (sentinel) keys placed after them in slot order.
// That moves every key a few times, where a radix sort over the 2 log2 V bits of the keys makes a
// pass a digit. No value is ever accumulated atomically: the runs are flagged, scanned and placed,
// and each entry's value is formed later from its run.
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include "ob_internal.cuh"

namespace ob {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ unsigned long long csr_key(int row, int col, int n) {
    const unsigned long long sentinel = (unsigned long long)n * (unsigned long long)n;
    if (row < 0 || row >= n || col < 0 || col >= n) return sentinel;
    return (unsigned long long)row * (unsigned long long)n + (unsigned long long)col;
}

// Tail slots: the sentinel (an unreferenced vertex keeps an empty row).
__global__ void fill_tail(unsigned long long* keys, long long tail, int n) {
    const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (v >= n) return;
    keys[tail + v] = (unsigned long long)n * (unsigned long long)n;
}

// One thread per face: both directions of the edge opposite each corner (slots 6 f + 2 e and
// + 1, payload 3 f + e: slot_payload), and the diagonal key of each in-range corner (every face
// writes the same key into a shared vertex's tail slot, so the race is benign).
__global__ void operator_keys(const int* __restrict__ faces, int n_faces, int n,
                              unsigned long long* __restrict__ keys) {
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
        const int v = c[e];
        if (v >= 0 && v < n) keys[tail + v] = csr_key(v, v, n);
    }
}

// The row of an in-range key row * n + col (< n^2, n < 2^31): the float64 quotient is within one of
// it (its relative error is 2^-53 and the quotient is below 2^31), and one step each way makes it
// exact -- the key's 64-bit integer division costs far more instructions than this.
__device__ __forceinline__ int key_row(unsigned long long key, int n) {
    long long r = (long long)((double)key / (double)n);
    const unsigned long long un = (unsigned long long)n;
    if ((unsigned long long)r * un > key) --r;
    else if ((unsigned long long)(r + 1) * un <= key) ++r;
    return (int)r;
}

// The payload of slot i: the corner 3 f + e of an edge slot 6 f + 2 e (+ 1), -1 for a tail slot.
__device__ __forceinline__ int slot_payload(long long i, long long tail) { return i < tail ? (int)(i / 2) : -1; }

// Row counts of the in-range keys (integer atomics: the counts, not their order, are used) and each
// slot's sentinel flag.
__global__ void row_counts(const unsigned long long* __restrict__ keys, long long count, unsigned long long sentinel,
                           int n, int* __restrict__ counts, int* __restrict__ sentinel_flag) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const unsigned long long key = keys[i];
    const bool inside = key < sentinel;
    sentinel_flag[i] = inside ? 0 : 1;
    if (inside) atomicAdd(&counts[key_row(key, n)], 1);
}

// Each in-range key into its row's bucket as (col << 32 | slot); each sentinel key to its place
// after every in-range one, in slot order.
__global__ void scatter_rows(const unsigned long long* __restrict__ keys, long long count, unsigned long long sentinel,
                             int n, const int* __restrict__ row_start, int* __restrict__ fill,
                             const int* __restrict__ sentinel_before, long long tail,
                             unsigned long long* __restrict__ bucket, unsigned long long* __restrict__ keys_out,
                             int* __restrict__ order_out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= count) return;
    const unsigned long long key = keys[i];
    if (key < sentinel) {
        const int row = key_row(key, n);
        const unsigned long long col = key - (unsigned long long)row * (unsigned long long)n;
        const int at = row_start[row] + atomicAdd(&fill[row], 1);
        bucket[at] = (col << 32) | (unsigned long long)i;
    } else {
        const long long at = (long long)row_start[n] + sentinel_before[i];
        keys_out[at] = key;
        order_out[at] = slot_payload(i, tail);
    }
}

// The sorted buckets back to keys and payloads, a group of 8 lanes a row.
__global__ void write_rows(const unsigned long long* __restrict__ sorted, const int* __restrict__ row_start, int n,
                           long long tail, unsigned long long* __restrict__ keys_out, int* __restrict__ order_out) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int row = (int)(t / 8), lane = (int)(t % 8);
    if (row >= n) return;
    for (int p = row_start[row] + lane; p < row_start[row + 1]; p += 8) {
        const unsigned long long v = sorted[p];
        keys_out[p] = (unsigned long long)row * (unsigned long long)n + (v >> 32);
        order_out[p] = slot_payload((long long)(v & 0xffffffffULL), tail);
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
    const int row = key_row(key, n);
    const int entry = inclusive[i] - 1;
    if (i == 0 || keys[i - 1] != key) {
        columns[entry] = (int)(key - (unsigned long long)row * (unsigned long long)n);
        run_start[entry] = (int)i;
        const int previous = (i == 0) ? -1 : key_row(keys[i - 1], n);
        for (int r = previous + 1; r <= row; ++r) offsets[r] = entry;
    }
    if (i + 1 == count || keys[i + 1] >= sentinel)
        for (int r = row + 1; r <= n; ++r) offsets[r] = inclusive[i];
}

struct PatternLayout {
    size_t keys_in = 0, sentinel_before = 0, flags = 0, bucket = 0, sorted = 0, counts = 0, starts = 0, fill = 0,
           sort_temp = 0, scan_temp = 0, total = 0;
};

int pattern_layout(int n, int n_faces, PatternLayout* out) {
    const long long count = 6LL * n_faces + n;
    PatternLayout l;
    size_t sort_bytes = 0, scan_bytes = 0, row_scan_bytes = 0;
    if (count > 0) {
        // The segmented sort's scratch depends on the in-range count, at most `count`.
        OB_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, sort_bytes, (const unsigned long long*)nullptr,
                                                   (unsigned long long*)nullptr, (int)count, std::max(n, 1),
                                                   (const int*)nullptr, (const int*)nullptr));
        OB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, (const int*)nullptr,
                                              (int*)nullptr, (int)count));
        OB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, row_scan_bytes, (const int*)nullptr, (int*)nullptr,
                                              n + 1));
        size_t sentinel_scan = 0;
        OB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, sentinel_scan, (const int*)nullptr, (int*)nullptr,
                                              (int)count));
        scan_bytes = std::max(std::max(scan_bytes, row_scan_bytes), sentinel_scan);
    }
    l.keys_in = 0;
    l.sentinel_before = align_up(l.keys_in + 8 * (size_t)count);
    l.flags = align_up(l.sentinel_before + 4 * (size_t)count);
    l.bucket = align_up(l.flags + 4 * (size_t)count);
    l.sorted = align_up(l.bucket + 8 * (size_t)count);
    l.counts = align_up(l.sorted + 8 * (size_t)count);
    l.starts = align_up(l.counts + 4 * (size_t)(n + 1));
    l.fill = align_up(l.starts + 4 * (size_t)(n + 1));
    l.sort_temp = align_up(l.fill + 4 * (size_t)(n + 1));
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
    auto* sentinel_before = reinterpret_cast<int*>(ws + l.sentinel_before);
    auto* flags = reinterpret_cast<int*>(ws + l.flags);
    auto* bucket = reinterpret_cast<unsigned long long*>(ws + l.bucket);
    auto* sorted = reinterpret_cast<unsigned long long*>(ws + l.sorted);
    auto* counts = reinterpret_cast<int*>(ws + l.counts);
    auto* starts = reinterpret_cast<int*>(ws + l.starts);
    auto* fill = reinterpret_cast<int*>(ws + l.fill);
    void* sort_temp = ws + l.sort_temp;
    void* scan_temp = ws + l.scan_temp;
    const long long tail = 6LL * n_faces;
    if (n_vertices > 0) {
        fill_tail<<<ceil_div(n_vertices, kThreads), kThreads, 0, stream>>>(keys_in, tail, n_vertices);
        OB_CHECK_LAUNCH("fill_tail");
    }
    if (n_faces > 0) {
        operator_keys<<<ceil_div(n_faces, kThreads), kThreads, 0, stream>>>(faces, n_faces, n_vertices, keys_in);
        OB_CHECK_LAUNCH("operator_keys");
    }
    const unsigned long long sentinel = (unsigned long long)n_vertices * n_vertices;
    auto* keys_out = reinterpret_cast<unsigned long long*>(keys);
    const int blocks = ceil_div(count, kThreads);
    size_t scan_bytes = l.total - 256 - l.scan_temp;
    OB_CUDA(cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)(n_vertices + 1), stream));
    OB_CUDA(cudaMemsetAsync(fill, 0, sizeof(int) * (size_t)(n_vertices + 1), stream));
    row_counts<<<blocks, kThreads, 0, stream>>>(keys_in, count, sentinel, std::max(n_vertices, 1), counts, flags);
    OB_CHECK_LAUNCH("row_counts");
    OB_CUDA(cub::DeviceScan::ExclusiveSum(scan_temp, scan_bytes, counts, starts, n_vertices + 1, stream));
    count_launch(1);
    // The sentinel slots' places among themselves.
    OB_CUDA(cub::DeviceScan::ExclusiveSum(scan_temp, scan_bytes, flags, sentinel_before, (int)count, stream));
    count_launch(1);
    scatter_rows<<<blocks, kThreads, 0, stream>>>(keys_in, count, sentinel, std::max(n_vertices, 1), starts, fill,
                                                  sentinel_before, tail, bucket, keys_out, order);
    OB_CHECK_LAUNCH("scatter_rows");
    if (n_vertices > 0) {
        // Sorted by (col, slot) within each row: the sort covers the in-range keys, starts[n] of them
        // (at most `count`, the size the scratch was sized for; the segments bound what is read).
        size_t sort_bytes = l.scan_temp - l.sort_temp;
        OB_CUDA(cub::DeviceSegmentedSort::SortKeys(sort_temp, sort_bytes, bucket, sorted, (int)count, n_vertices,
                                                   starts, starts + 1, stream));
        count_launch(1);
        write_rows<<<ceil_div(8LL * n_vertices, kThreads), kThreads, 0, stream>>>(sorted, starts, n_vertices, tail,
                                                                                 keys_out, order);
        OB_CHECK_LAUNCH("write_rows");
    }
    run_flags<<<blocks, kThreads, 0, stream>>>(reinterpret_cast<unsigned long long*>(keys), count,
                                               sentinel, flags);
    OB_CHECK_LAUNCH("run_flags");
    OB_CUDA(cub::DeviceScan::InclusiveSum(scan_temp, scan_bytes, flags, flags, (int)count, stream));
    count_launch(1);
    place_runs<<<blocks, kThreads, 0, stream>>>(reinterpret_cast<unsigned long long*>(keys), flags,
                                                count, sentinel, n_vertices, offsets, columns,
                                                run_start);
    OB_CHECK_LAUNCH("place_runs");
    return OB_OK;
}

}  // extern "C"
