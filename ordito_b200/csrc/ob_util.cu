// Small utilities the host layer needs so that no value is formed on the host.
#include "ob_internal.cuh"
#include "ob_scratch.cuh"

namespace ob {
namespace {

template <typename S, typename T>
__global__ void cast_scale_kernel(long long n, const S* __restrict__ in, T* __restrict__ out,
                                  double scale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (T)((double)in[i] * scale);
}

// Axis-aligned bounds of float32 points: out = (min x, min y, min z, max x, max y, max z).
__global__ void bounds_kernel(const float* __restrict__ xyz, int n, float* __restrict__ partials,
                              unsigned int* counter, double* __restrict__ out) {
    __shared__ float scratch[32];
    __shared__ int last;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int d = 0; d < 3; ++d) {
            const float v = xyz[3 * i + d];
            lo[d] = fminf(lo[d], v);
            hi[d] = fmaxf(hi[d], v);
        }
    for (int d = 0; d < 3; ++d) {
        const float a = -block_max(-lo[d], scratch, -INFINITY);
        const float b = block_max(hi[d], scratch, -INFINITY);
        if (threadIdx.x == 0) {
            partials[6 * blockIdx.x + d] = a;
            partials[6 * blockIdx.x + 3 + d] = b;
        }
    }
    if (!last_block_arrived(counter, &last)) return;
    if (threadIdx.x != 0) return;
    for (int d = 0; d < 3; ++d) {
        float a = INFINITY, b = -INFINITY;
        for (int bx = 0; bx < (int)gridDim.x; ++bx) {
            a = fminf(a, __ldcg(&partials[6 * bx + d]));
            b = fmaxf(b, __ldcg(&partials[6 * bx + 3 + d]));
        }
        out[d] = a;
        out[3 + d] = b;
    }
}

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_bounds(const float* xyz, int n, double* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(out != nullptr && n >= 0, "ob_bounds: bad argument");
    if (n == 0) {
        const double empty[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        OB_CUDA(cudaMemcpyAsync(out, empty, sizeof(empty), cudaMemcpyHostToDevice, stream));
        OB_CUDA(cudaStreamSynchronize(stream));
        return OB_OK;
    }
    OB_REQUIRE(xyz != nullptr, "ob_bounds: null points");
    const int blocks = std::max(1, std::min(ceil_div(n, 256), 2 * sm_count()));
    Scratch scratch(stream);
    float* partials = scratch.take<float>(6 * (size_t)blocks);
    unsigned int* counter = scratch.take<unsigned int>(1);
    int st = scratch.commit();
    if (st) return st;
    OB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned int), stream));
    bounds_kernel<<<blocks, 256, 0, stream>>>(xyz, n, partials, counter, out);
    OB_CHECK_LAUNCH("bounds");
    return OB_OK;
}

// out[i] = (dst type)(in[i] * scale); types: 0 float32, 1 float64.
int ob_cast_scale(const void* in, int in_type, void* out, int out_type, long long n, double scale,
                  ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    if (n <= 0) return OB_OK;
    OB_REQUIRE(in && out, "ob_cast_scale: null pointer");
    OB_REQUIRE((in_type == 0 || in_type == 1) && (out_type == 0 || out_type == 1),
               "ob_cast_scale: types are 0 (float32) or 1 (float64)");
    const int blocks = (int)std::min((n + 255) / 256, (long long)8 * sm_count());
    if (in_type == 0 && out_type == 0)
        cast_scale_kernel<<<blocks, 256, 0, stream>>>(n, (const float*)in, (float*)out, scale);
    else if (in_type == 0 && out_type == 1)
        cast_scale_kernel<<<blocks, 256, 0, stream>>>(n, (const float*)in, (double*)out, scale);
    else if (in_type == 1 && out_type == 0)
        cast_scale_kernel<<<blocks, 256, 0, stream>>>(n, (const double*)in, (float*)out, scale);
    else
        cast_scale_kernel<<<blocks, 256, 0, stream>>>(n, (const double*)in, (double*)out, scale);
    OB_CHECK_LAUNCH("cast_scale");
    return OB_OK;
}

}  // extern "C"
