// The marched settled solve: A x = b band by band, every entry to its own relative precision.
//
// The fallback of the settled heat solve where the operator's factorisation is refused
// (ordito/linalg.py:2765 _march_settled, the kernels of ordito/kernels/linalg.py:1229-1545). A
// heat solution decays over hundreds of e-folds, below any normwise solve's round-off; the march
// solves it a band at a time, outward from the right-hand side's support. A band is the rows not
// yet finished within `hops` hops of the finished ones (of the support, at first), grown breadth
// first a hop a launch; its system is the operator's band-by-band block with the finished
// neighbours' values moved to the right-hand side (Dirichlet data) and zero beyond it, the whole
// divided by the largest datum so the front is O(1). It is solved by float64 CG to a relative
// residual of 1e-14; rows both resolved (>= e^-14 of the band's peak) and clear of the zero the
// band stands on (>= e^16 times its outer layer) are finished, as is a row far below a neighbour
// (a sign change, e^4 past the threshold); every row's value seeds the next band's guess. The
// next band's hop count is rescaled from this band's span in e-folds toward 14 + 16.
//
// Differences from the reference, by design: the band's rows are always sorted (the reference
// sorts them only under its deterministic mode), so the band system is in the operator's order
// and the result is the same on every run; band solves use this library's float64 CG (Jacobi,
// or the Jacobi-Chebyshev polynomial from 2^17 rows where the reference escalates to a V-cycle).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ob_internal.cuh"

namespace ob {
namespace {

constexpr double kResolved = 14.0;           // ordito/linalg.py:188 _MARCH_RESOLVED
constexpr double kMargin = 16.0;             // :189 _MARCH_MARGIN
constexpr double kTolerance = 1e-14;         // :190 _MARCH_TOLERANCE
const double kDominated = std::exp(4.0);     // :193 _MARCH_DOMINATED
constexpr int kFirstHops = 32;               // :197 _MARCH_FIRST_HOPS
constexpr int kGrowth = 4;                   // :198 _MARCH_GROWTH
constexpr int kPolynomialFrom = 1 << 17;     // :203 _MARCH_MULTIGRID_FROM (see the header note)
constexpr int kMaxBands = 20000;             // a bound on the loop (each band finishes rows)
constexpr int kThreads = 256;

enum Word { kScale = 0, kPeak = 1, kOuter = 2, kHasOuter = 3, kWords = 4 };

// atomicMax on a non-negative double: its bits order as an unsigned integer's.
__device__ __forceinline__ void raise_to(double* word, double value) {
    if (!(value > *word)) return;
    atomicMax(reinterpret_cast<unsigned long long*>(word), __double_as_longlong(value));
}

__device__ __forceinline__ void append(int v, int* local, int* band, int* count) {
    const int slot = atomicAdd(count, 1);
    local[v] = slot;
    band[slot] = v;
}

__global__ void seed_support_kernel(int n, const double* __restrict__ rhs, int* local, int* band,
                                    int* count) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n && rhs[v] != 0.0) append(v, local, band, count);
}

__global__ void seed_front_kernel(int n, const int* __restrict__ offsets, const int* __restrict__ columns,
                                  const int* __restrict__ finished, int* local, int* band, int* count) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n || finished[v]) return;
    for (int e = offsets[v]; e < offsets[v + 1]; ++e)
        if (finished[columns[e]]) {
            append(v, local, band, count);
            return;
        }
}

__global__ void close_hop_kernel(const int* count, int hop, int* bounds) { bounds[hop] = *count; }

// Hop `hop` of the breadth-first growth: every unfinished neighbour of the last hop's rows not yet
// in the band joins it, claimed by a compare-and-swap so it is appended once. Lanes stride the
// hop's rows (its length is on the device only).
__global__ void expand_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                              const int* __restrict__ finished, const int* __restrict__ bounds, int hop,
                              int* local, int* band, int* count) {
    const int end = bounds[hop];
    for (int i = bounds[hop - 1] + blockIdx.x * blockDim.x + threadIdx.x; i < end;
         i += gridDim.x * blockDim.x) {
        const int v = band[i];
        for (int e = offsets[v]; e < offsets[v + 1]; ++e) {
            const int j = columns[e];
            if (finished[j] == 0 && local[j] == -1 && atomicCAS(&local[j], -1, -2) == -1)
                append(j, local, band, count);
        }
    }
}

__global__ void renumber_kernel(int m, const int* __restrict__ band, int* local) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) local[band[i]] = i;
}

// A band row's in-band entry count (into counts[i]) and the band's scale: the largest datum it
// reads (a right-hand-side entry or a finished neighbour's value).
__global__ void band_rows_kernel(int m, const int* __restrict__ offsets, const int* __restrict__ columns,
                                 const int* __restrict__ band, const int* __restrict__ local,
                                 const int* __restrict__ finished, const double* __restrict__ solution,
                                 const double* __restrict__ rhs, int* counts, double* words) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int v = band[i];
    int count = 0;
    double top = fabs(rhs[v]);
    for (int e = offsets[v]; e < offsets[v + 1]; ++e) {
        const int j = columns[e];
        if (local[j] >= 0) ++count;
        else if (finished[j]) top = fmax(top, fabs(solution[j]));
    }
    counts[i] = count;
    raise_to(&words[kScale], top);
}

// The band system's row i: in-band entries renumbered, finished neighbours' terms moved to the
// right-hand side, divided by the band's scale; the guess is the last band's value there.
__global__ void band_system_kernel(int m, const int* __restrict__ offsets, const int* __restrict__ columns,
                                   const double* __restrict__ values, const int* __restrict__ band,
                                   const int* __restrict__ local, const int* __restrict__ finished,
                                   const double* __restrict__ solution, const double* __restrict__ rhs,
                                   const double* __restrict__ tentative, const double* __restrict__ words,
                                   const int* __restrict__ band_offsets, int* out_columns,
                                   double* out_values, double* out_rhs, double* out_guess) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int v = band[i];
    int slot = band_offsets[i];
    double r = rhs[v];
    for (int e = offsets[v]; e < offsets[v + 1]; ++e) {
        const int j = columns[e];
        const int lj = local[j];
        if (lj >= 0) {
            out_columns[slot] = lj;
            out_values[slot] = values[e];
            ++slot;
        } else if (finished[j]) {
            r -= values[e] * solution[j];
        }
    }
    const double scale = words[kScale];
    const double inverse = scale > 0.0 ? 1.0 / scale : 0.0;
    out_rhs[i] = r * inverse;
    out_guess[i] = tentative[v] * inverse;
}

// The band solution's peak magnitude and its peak over the outer layer (rows with an unfinished
// neighbour outside the band, where the zero beyond stands in for the field).
__global__ void band_extremes_kernel(int m, const int* __restrict__ offsets, const int* __restrict__ columns,
                                     const int* __restrict__ band, const int* __restrict__ local,
                                     const int* __restrict__ finished, const double* __restrict__ x,
                                     double* words) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int v = band[i];
    const double magnitude = fabs(x[i]);
    raise_to(&words[kPeak], magnitude);
    for (int e = offsets[v]; e < offsets[v + 1]; ++e) {
        const int j = columns[e];
        if (local[j] < 0 && !finished[j]) {
            raise_to(&words[kOuter], magnitude);
            raise_to(&words[kHasOuter], 1.0);
            return;
        }
    }
}

// Finish the rows at `threshold` or above, and a row far below a neighbour (in the band or
// finished, at the band's scale) at `dominated` or above; every row's value seeds the next guess.
__global__ void band_commit_kernel(int m, const int* __restrict__ offsets, const int* __restrict__ columns,
                                   const int* __restrict__ band, const int* __restrict__ local,
                                   const int* __restrict__ finished, const double* __restrict__ x,
                                   const double* __restrict__ words, double threshold, double dominated,
                                   double* solution, double* tentative, int* keep) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int v = band[i];
    const double scale = words[kScale];
    int kept = fabs(x[i]) >= threshold;
    if (!kept) {
        const double inverse = scale > 0.0 ? 1.0 / scale : 0.0;
        for (int e = offsets[v]; e < offsets[v + 1] && !kept; ++e) {
            const int j = columns[e];
            const int lj = local[j];
            if (lj >= 0) kept = fabs(x[lj]) >= dominated;
            else if (finished[j]) kept = fabs(solution[j]) * inverse >= dominated;
        }
    }
    const double value = x[i] * scale;
    tentative[v] = value;
    if (kept) solution[v] = value;
    keep[i] = kept;
}

__global__ void band_release_kernel(int m, const int* __restrict__ band, const int* __restrict__ keep,
                                    int* local, int* finished) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int v = band[i];
    local[v] = -1;
    if (keep[i]) finished[v] = 1;
}

__global__ void fill_int_kernel(long long n, int* out, int value) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x)
        out[t] = value;
}

struct Buffers {
    std::vector<void*> owned;
    cudaStream_t stream;
    ~Buffers() {
        for (void* p : owned) cudaFreeAsync(p, stream);
    }
    template <typename T>
    int take(T** p, size_t n) {
        void* q = nullptr;
        const cudaError_t e = pool_malloc(&q, sizeof(T) * std::max<size_t>(n, 1), stream);
        if (e != cudaSuccess) return cuda_status(e, "ob_march_solve: allocation");
        owned.push_back(q);
        *p = static_cast<T*>(q);
        return OB_OK;
    }
};

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_march_solve(int n, const int32_t* offsets, const int32_t* columns, const double* values,
                   const double* rhs, double* x, long long* info, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n >= 1 && offsets && columns && values && rhs && x, "ob_march_solve: bad argument");
    int nnz_total = 0;
    OB_CUDA(cudaMemcpyAsync(&nnz_total, offsets + n, sizeof(int), cudaMemcpyDeviceToHost, stream));
    OB_CUDA(cudaStreamSynchronize(stream));
    Buffers buf;
    buf.stream = stream;
    int *finished, *local, *band, *sorted, *count, *bounds, *counts, *band_offsets, *band_columns, *keep;
    double *tentative, *words, *band_values, *band_rhs, *band_x;
    int st;
    if ((st = buf.take(&finished, n)) || (st = buf.take(&local, n)) || (st = buf.take(&band, n)) ||
        (st = buf.take(&sorted, n)) || (st = buf.take(&count, 1)) || (st = buf.take(&counts, n + 1)) ||
        (st = buf.take(&band_offsets, n + 1)) || (st = buf.take(&band_columns, nnz_total)) ||
        (st = buf.take(&keep, n)) || (st = buf.take(&tentative, n)) || (st = buf.take(&words, kWords)) ||
        (st = buf.take(&band_values, nnz_total)) || (st = buf.take(&band_rhs, n)) ||
        (st = buf.take(&band_x, n)))
        return st;
    size_t sort_bytes = 0, scan_bytes = 0;
    OB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, band, sorted, n));
    OB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, counts, band_offsets, n + 1));
    void* temp = nullptr;
    if ((st = buf.take(reinterpret_cast<char**>(&temp), std::max(sort_bytes, scan_bytes)))) return st;
    const int grid = ceil_div(n, kThreads);
    OB_CUDA(cudaMemsetAsync(finished, 0, sizeof(int) * n, stream));
    OB_CUDA(cudaMemsetAsync(tentative, 0, sizeof(double) * n, stream));
    OB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, stream));
    fill_int_kernel<<<grid, kThreads, 0, stream>>>(n, local, -1);
    OB_CHECK_LAUNCH("march fill");
    const double resolved = std::exp(-kResolved), margin = std::exp(kMargin);
    const double span_target = kResolved + kMargin;
    int hops = kFirstHops;
    bool started = false;
    long long rounds = 0, bands = 0, committed = 0;
    int whole = -1;
    std::vector<int> bounds_host;
    std::vector<int> zero_bounds;
    int* hop_bounds = nullptr;
    int hop_capacity = 0;
    const int expand_grid = std::max(1, std::min(ceil_div(n, kThreads), 8 * sm_count()));
    for (;;) {
        if (++bands > kMaxBands) return fail(OB_ERR_NOT_CONVERGED, "ob_march_solve: band limit reached");
        if (hops + 2 > hop_capacity) {
            hop_capacity = 2 * (hops + 2);
            if ((st = buf.take(&hop_bounds, hop_capacity))) return st;
        }
        OB_CUDA(cudaMemsetAsync(count, 0, sizeof(int), stream));
        OB_CUDA(cudaMemsetAsync(hop_bounds, 0, sizeof(int) * (hops + 2), stream));
        if (started)
            seed_front_kernel<<<grid, kThreads, 0, stream>>>(n, offsets, columns, finished, local, band, count);
        else
            seed_support_kernel<<<grid, kThreads, 0, stream>>>(n, rhs, local, band, count);
        OB_CHECK_LAUNCH("march seed");
        close_hop_kernel<<<1, 1, 0, stream>>>(count, 1, hop_bounds);
        OB_CHECK_LAUNCH("march close hop");
        for (int hop = 1; hop <= hops; ++hop) {
            expand_kernel<<<expand_grid, kThreads, 0, stream>>>(offsets, columns, finished, hop_bounds, hop,
                                                                local, band, count);
            OB_CHECK_LAUNCH("march expand");
            close_hop_kernel<<<1, 1, 0, stream>>>(count, hop + 1, hop_bounds);
            OB_CHECK_LAUNCH("march close hop");
        }
        int m = 0;
        OB_CUDA(cudaMemcpyAsync(&m, count, sizeof(int), cudaMemcpyDeviceToHost, stream));
        OB_CUDA(cudaStreamSynchronize(stream));
        if (m == 0 || m == whole) break;
        // Sorted, the band's rows are numbered as the operator's are.
        size_t bytes = sort_bytes;
        OB_CUDA(cub::DeviceRadixSort::SortKeys(temp, bytes, band, sorted, m, 0, 32, stream));
        count_launch();
        OB_CUDA(cudaMemcpyAsync(band, sorted, sizeof(int) * m, cudaMemcpyDeviceToDevice, stream));
        const int mg = ceil_div(m, kThreads);
        renumber_kernel<<<mg, kThreads, 0, stream>>>(m, band, local);
        OB_CHECK_LAUNCH("march renumber");
        OB_CUDA(cudaMemsetAsync(words, 0, sizeof(double) * kWords, stream));
        OB_CUDA(cudaMemsetAsync(counts + m, 0, sizeof(int), stream));
        band_rows_kernel<<<mg, kThreads, 0, stream>>>(m, offsets, columns, band, local, finished, x, rhs,
                                                      counts, words);
        OB_CHECK_LAUNCH("march band rows");
        bytes = scan_bytes;
        OB_CUDA(cub::DeviceScan::ExclusiveSum(temp, bytes, counts, band_offsets, m + 1, stream));
        count_launch();
        band_system_kernel<<<mg, kThreads, 0, stream>>>(m, offsets, columns, values, band, local, finished, x,
                                                        rhs, tentative, words, band_offsets, band_columns,
                                                        band_values, band_rhs, band_x);
        OB_CHECK_LAUNCH("march band system");
        // The band solve: float64 CG to a relative residual of 1e-14 from the last band's values.
        void* solver = nullptr;
        st = ob_pcg_create(m, band_offsets, band_columns, band_values, 1, m >= kPolynomialFrom ? 1 : 0, 0,
                           &solver, stream);
        if (st) return st;
        int iterations = 0;
        double residual = 0.0;
        st = ob_pcg_solve(solver, band_rhs, band_x, kTolerance, 10 * m, &iterations, &residual, stream);
        ob_pcg_destroy(solver);
        if (st) return st;
        rounds += iterations;
        band_extremes_kernel<<<mg, kThreads, 0, stream>>>(m, offsets, columns, band, local, finished, band_x,
                                                          words);
        OB_CHECK_LAUNCH("march band extremes");
        double w[kWords];
        OB_CUDA(cudaMemcpyAsync(w, words, sizeof(w), cudaMemcpyDeviceToHost, stream));
        OB_CUDA(cudaStreamSynchronize(stream));
        const double peak = w[kPeak];
        double outer = w[kOuter];
        const bool has_outer = w[kHasOuter] > 0.0;
        double threshold = resolved * peak;
        if (has_outer) {
            // An outer layer the solve left below its own tolerance of the peak is unresolved.
            outer = std::max(outer, kTolerance * peak);
            threshold = std::max(threshold, margin * outer);
            const double span = peak > outer ? std::log(peak / outer) : 0.0;
            const long long target = span <= 0.0 ? (long long)hops * kGrowth
                                                 : (long long)std::ceil(hops * span_target / span);
            hops = (int)std::min<long long>({(long long)hops * kGrowth,
                                             std::max<long long>({(long long)hops / 2, target, 1LL}),
                                             (long long)n});
        }
        band_commit_kernel<<<mg, kThreads, 0, stream>>>(m, offsets, columns, band, local, finished, band_x,
                                                        words, threshold, threshold * kDominated, x,
                                                        tentative, keep);
        OB_CHECK_LAUNCH("march band commit");
        band_release_kernel<<<mg, kThreads, 0, stream>>>(m, band, keep, local, finished);
        OB_CHECK_LAUNCH("march band release");
        committed += m;
        started = started || peak >= threshold;
        whole = has_outer ? -1 : m;
    }
    if (info) {
        info[0] = bands;
        info[1] = rounds;
        info[2] = committed;
    }
    OB_CUDA(cudaStreamSynchronize(stream));
    return OB_OK;
}

}  // extern "C"
