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

__global__ void floor_kernel(long long n, float* __restrict__ values, float floor) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        values[i] = fmaxf(values[i], floor);
}

__global__ void axpby_kernel(long long n, double a, const double* __restrict__ x, double b,
                             const double* y, double* out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = a * x[i] + b * y[i];
}

// out[c][r] = in[r][c] for a rows x cols row-major float64 matrix.
__global__ void transpose_kernel(int rows, int cols, const double* __restrict__ in,
                                 double* __restrict__ out) {
    __shared__ double tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[i][threadIdx.x] = in[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[threadIdx.x][i];
    }
}

// Source indicators of several columns: u0[v][c] = 1 for v in column c's sources.
__global__ void seed_columns_kernel(const int* __restrict__ sources,
                                    const int* __restrict__ source_offsets, int n_columns, int n,
                                    double* __restrict__ u0, int* __restrict__ invalid) {
    const int c = blockIdx.y;
    const int begin = source_offsets[c], end = source_offsets[c + 1];
    for (int i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end;
         i += gridDim.x * blockDim.x) {
        const int v = sources[i];
        if (v < 0 || v >= n) {
            invalid[0] = 1;
            continue;
        }
        u0[(size_t)v * n_columns + c] = 1.0;
    }
}

// Eight independent float64 FMA chains per thread: the device's FP64 FMA throughput.
__global__ void fp64_fma_kernel(int iterations, double seed, double* __restrict__ sink) {
    double a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = seed + threadIdx.x + j;
    const double m = 0.999999, c = 1e-7;
    for (int i = 0; i < iterations; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = fma(a[j], m, c);
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += a[j];
    if (s == 12345.678) sink[0] = s;  // keeps the chains live
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

int ob_fp64_peak(float* tflops, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(tflops != nullptr, "ob_fp64_peak: null output");
    Scratch scratch(stream);
    double* sink = scratch.take<double>(1);
    int st = scratch.commit();
    if (st) return st;
    const int blocks = 8 * sm_count(), threads = 256, iterations = 4096;
    cudaEvent_t start, end;
    OB_CUDA(cudaEventCreate(&start));
    OB_CUDA(cudaEventCreate(&end));
    fp64_fma_kernel<<<blocks, threads, 0, stream>>>(iterations, 1.0, sink);  // warm-up
    cudaEventRecord(start, stream);
    for (int r = 0; r < 5; ++r) fp64_fma_kernel<<<blocks, threads, 0, stream>>>(iterations, 1.0, sink);
    cudaEventRecord(end, stream);
    count_launch(6);
    cudaError_t e = cudaEventSynchronize(end);
    float ms = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, start, end);
    cudaEventDestroy(start);
    cudaEventDestroy(end);
    if (e != cudaSuccess) return cuda_status(e, "ob_fp64_peak");
    const double flops = 5.0 * blocks * threads * (double)iterations * 8.0 * 2.0;
    *tflops = (float)(flops / (ms * 1e-3) / 1e12);
    return OB_OK;
}

int ob_axpby(long long n, double a, const double* x, double b, const double* y, double* out,
             ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    if (n <= 0) return OB_OK;
    OB_REQUIRE(x && y && out, "ob_axpby: null pointer");
    const int blocks = (int)std::min((n + 255) / 256, (long long)8 * sm_count());
    axpby_kernel<<<blocks, 256, 0, stream>>>(n, a, x, b, y, out);
    OB_CHECK_LAUNCH("axpby");
    return OB_OK;
}

int ob_transpose(int rows, int cols, const double* in, double* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    if (rows <= 0 || cols <= 0) return OB_OK;
    OB_REQUIRE(in && out && in != out, "ob_transpose: bad argument");
    transpose_kernel<<<dim3(ceil_div(cols, 32), ceil_div(rows, 32)), dim3(32, 8), 0, stream>>>(
        rows, cols, in, out);
    OB_CHECK_LAUNCH("transpose");
    return OB_OK;
}

int ob_seed_columns(const int32_t* sources, const int32_t* source_offsets, int n_columns,
                    int n_vertices, double* u0, int32_t* invalid, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_columns >= 1 && n_vertices >= 0 && invalid && source_offsets,
               "ob_seed_columns: bad argument");
    OB_CUDA(cudaMemsetAsync(invalid, 0, sizeof(int32_t), stream));
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(u0 && sources, "ob_seed_columns: null pointer");
    OB_CUDA(cudaMemsetAsync(u0, 0, sizeof(double) * (size_t)n_vertices * n_columns, stream));
    seed_columns_kernel<<<dim3(1, n_columns), 128, 0, stream>>>(sources, source_offsets, n_columns,
                                                              n_vertices, u0, invalid);
    OB_CHECK_LAUNCH("seed_columns");
    return OB_OK;
}

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

int ob_floor_f32(float* values, long long n, float floor, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    if (n <= 0) return OB_OK;
    OB_REQUIRE(values, "ob_floor_f32: null pointer");
    const int blocks = (int)std::min((n + 255) / 256, (long long)8 * sm_count());
    floor_kernel<<<blocks, 256, 0, stream>>>(n, values, floor);
    OB_CHECK_LAUNCH("floor");
    return OB_OK;
}

}  // extern "C"
