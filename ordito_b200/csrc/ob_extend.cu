// f3: extend_scalar's device steps (ordito/heat.py:2321 extend_scalar, :2426 _extend_scalar;
// kernels/heat.py:3858 seed_source_scalars, :3933 extend_from_ratio).
//
// Two right-hand sides diffuse through the heat system as one two-column solve: an indicator of
// where the sources are and the values they carry. Their quotient stays near the nearest
// source's value (both fall off at the same rate away from the sources). The range check measures
// how far the quotient leaves the source values' range where the indicator is non-zero.
#include <cfloat>

#include "ob_internal.cuh"

namespace ob {
namespace {

constexpr int kThreads = 256;

// rhs[v][0] += 1 and rhs[v][1] += value for each source (rhs zeroed before); an index outside
// [0, n) sets invalid[0].
__global__ void extend_seed_kernel(const int* __restrict__ sources, const double* __restrict__ values, int k,
                                   int n, double* __restrict__ rhs, int* __restrict__ invalid) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= k) return;
    const int v = sources[s];
    if (v < 0 || v >= n) {
        *invalid = 1;
        return;
    }
    atomicAdd(rhs + 2 * (size_t)v, 1.0);
    atomicAdd(rhs + 2 * (size_t)v + 1, values[s]);
}

// range[0] = min and range[1] = max of the source values (one block, a fixed tree).
__global__ void extend_value_range_kernel(const double* __restrict__ values, int k, double* __restrict__ range) {
    __shared__ double scratch[32];
    double lo = DBL_MAX, hi = -DBL_MAX;
    for (int s = threadIdx.x; s < k; s += blockDim.x) {
        lo = fmin(lo, values[s]);
        hi = fmax(hi, values[s]);
    }
    lo = -block_max(-lo, scratch, -DBL_MAX);
    hi = block_max(hi, scratch, -DBL_MAX);
    if (threadIdx.x == 0) {
        range[0] = lo;
        range[1] = hi;
    }
}

// extended[i] = weighted / indicator (0 where the indicator is exactly 0), and the largest
// excess over [range[0], range[1]] where it is not, folded by an unsigned maximum of the
// non-negative excess's bits (their order is the values') into excess_bits.
__global__ void extend_ratio_kernel(const double* __restrict__ diffused, int n, const double* __restrict__ range,
                                    double* __restrict__ extended, unsigned long long* __restrict__ excess_bits) {
    __shared__ double scratch[32];
    const double lo = range[0], hi = range[1];
    double excess = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double indicator = diffused[2 * (size_t)i], weighted = diffused[2 * (size_t)i + 1];
        const double value = indicator != 0.0 ? weighted / indicator : 0.0;
        extended[i] = value;
        if (indicator != 0.0) excess = fmax(excess, fmax(value - hi, lo - value));
    }
    excess = block_max(excess, scratch, 0.0);
    if (threadIdx.x == 0 && excess > 0.0) atomicMax(excess_bits, (unsigned long long)__double_as_longlong(excess));
}

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_extend_seed(const int32_t* sources, const double* values, int n_sources, int n_vertices, double* rhs,
                   double* range, int32_t* invalid, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_sources >= 1 && n_vertices >= 1, "ob_extend_seed: bad size");
    OB_REQUIRE(sources && values && rhs && range && invalid, "ob_extend_seed: null pointer");
    OB_CUDA(cudaMemsetAsync(rhs, 0, sizeof(double) * 2 * (size_t)n_vertices, stream));
    OB_CUDA(cudaMemsetAsync(invalid, 0, sizeof(int32_t), stream));
    OB_CUDA(cudaMemsetAsync(range, 0, 3 * sizeof(double), stream));
    extend_seed_kernel<<<ceil_div(n_sources, kThreads), kThreads, 0, stream>>>(sources, values, n_sources, n_vertices,
                                                                               rhs, invalid);
    OB_CHECK_LAUNCH("extend seed");
    extend_value_range_kernel<<<1, kThreads, 0, stream>>>(values, n_sources, range);
    OB_CHECK_LAUNCH("extend value range");
    return OB_OK;
}

int ob_extend_ratio(const double* diffused, int n_vertices, double* range, double* extended, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 1, "ob_extend_ratio: bad size");
    OB_REQUIRE(diffused && range && extended, "ob_extend_ratio: null pointer");
    const int blocks = std::max(1, std::min(ceil_div(n_vertices, kThreads), 4 * sm_count()));
    extend_ratio_kernel<<<blocks, kThreads, 0, stream>>>(diffused, n_vertices, range, extended,
                                                         reinterpret_cast<unsigned long long*>(range + 2));
    OB_CHECK_LAUNCH("extend ratio");
    return OB_OK;
}

}  // extern "C"
