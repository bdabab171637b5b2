// a6, a8, a13: the per-query kernels -- source indicator, unit-gradient divergence and the shift.
#include "ob_geometry.cuh"
#include "ob_internal.cuh"
#include "ob_scratch.cuh"

namespace ob {
namespace {

constexpr int kThreads = 256;

// ordito/kernels/heat.py:600-623 (flag_out_of_range, seed_source_indicator).
__global__ void seed_kernel(const int* __restrict__ sources, int k, int n, double* __restrict__ u0,
                            int* __restrict__ invalid) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= k) return;
    const int v = sources[t];
    if (v < 0 || v >= n) {
        invalid[0] = 1;
        return;
    }
    u0[v] = 1.0;
}

struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 widen(f3 a) { return d3{(double)a.x, (double)a.y, (double)a.z}; }
__device__ __forceinline__ d3 dsub(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 dcross(d3 a, d3 b) {
    return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// ordito/kernels/triangles.py:834-894 (face_gradient_given, face_unit_gradient),
// kernels/predicates.py:719-724 (stable_normalize) and kernels/heat.py:626-687
// (accumulate_face_divergence, unit_gradient_divergence). One thread per (face, column): the
// float64 gradient of u in the face plane, scaled by its largest component and normalised, then
// the cotangent-weighted divergence terms added into the face's three vertices. Integrating the
// gradient direction (not its negation) accumulates -div(X) directly.
__global__ void grad_div_kernel(const float* __restrict__ xyz, const int* __restrict__ faces,
                                int n_faces, const float* __restrict__ normals,
                                const float* __restrict__ areas, const double* __restrict__ u,
                                const float* __restrict__ cot, int k,
                                double* __restrict__ neg_div) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n_faces * k) return;
    const int f = (int)(t / k), c = (int)(t % k);
    const int i0 = faces[3 * f], i1 = faces[3 * f + 1], i2 = faces[3 * f + 2];
    const d3 v0 = widen(load_f3(xyz, i0)), v1 = widen(load_f3(xyz, i1)), v2 = widen(load_f3(xyz, i2));
    const d3 n = widen(load_f3(normals, f));
    const double area = (double)areas[f];
    d3 g{0.0, 0.0, 0.0};
    if (area > 0.0) {
        const double u0 = u[(size_t)i0 * k + c], u1 = u[(size_t)i1 * k + c],
                     u2 = u[(size_t)i2 * k + c];
        const d3 a = dcross(n, dsub(v2, v1)), b = dcross(n, dsub(v0, v2)), e = dcross(n, dsub(v1, v0));
        const double inv = 2.0 * area;
        g = d3{(u0 * a.x + u1 * b.x + u2 * e.x) / inv, (u0 * a.y + u1 * b.y + u2 * e.y) / inv,
               (u0 * a.z + u1 * b.z + u2 * e.z) / inv};
    }
    const double largest = fmax(fabs(g.x), fmax(fabs(g.y), fabs(g.z)));
    d3 x{0.0, 0.0, 0.0};
    if (largest != 0.0) {
        const d3 w{g.x / largest, g.y / largest, g.z / largest};
        const double len = sqrt(ddot(w, w));
        if (len > 0.0) x = d3{w.x / len, w.y / len, w.z / len};
    }
    const double c0 = (double)cot[3 * f], c1 = (double)cot[3 * f + 1], c2 = (double)cot[3 * f + 2];
    const double d0 = c2 * ddot(dsub(v1, v0), x) + c1 * ddot(dsub(v2, v0), x);
    const double d1 = c0 * ddot(dsub(v2, v1), x) + c2 * ddot(dsub(v0, v1), x);
    const double d2 = c1 * ddot(dsub(v0, v2), x) + c0 * ddot(dsub(v1, v2), x);
    atomicAdd(&neg_div[(size_t)i0 * k + c], d0);
    atomicAdd(&neg_div[(size_t)i1 * k + c], d1);
    atomicAdd(&neg_div[(size_t)i2 * k + c], d2);
}

// ordito/kernels/heat.py:3383-3403 (source_and_global_sums): per column, the sum of phi over its
// sources and over every vertex. Grid (blocks, columns); block partials folded in block order by
// the last block of the whole launch.
__global__ void source_sums_kernel(const double* __restrict__ phi, int n,
                                   const int* __restrict__ sources,
                                   const int* __restrict__ source_offsets, int n_sources, int k,
                                   double2* __restrict__ partials, unsigned int* counter,
                                   double2* __restrict__ sums) {
    __shared__ double scratch[32];
    __shared__ int last;
    const int c = blockIdx.y;
    const int s_begin = source_offsets ? source_offsets[c] : 0;
    const int s_end = source_offsets ? source_offsets[c + 1] : n_sources;
    double at_sources = 0.0, everywhere = 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s_end - s_begin; i += stride)
        at_sources += phi[(size_t)sources[s_begin + i] * k + c];
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        everywhere += phi[(size_t)v * k + c];
    const double a = block_sum(at_sources, scratch);
    const double b = block_sum(everywhere, scratch);
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

// ordito/kernels/heat.py:3406-3424 (shift_and_orient).
__global__ void shift_kernel(double* __restrict__ phi, int n, const double2* __restrict__ sums,
                             const int* __restrict__ source_offsets, int n_sources, int k,
                             int orient) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * k) return;
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

int ob_seed(const int32_t* sources, int n_sources, int n_vertices, double* u0, int32_t* invalid,
            ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_sources >= 0 && n_vertices >= 0, "ob_seed: negative size");
    OB_REQUIRE(invalid != nullptr, "ob_seed: null invalid flag");
    OB_CUDA(cudaMemsetAsync(invalid, 0, sizeof(int32_t), stream));
    if (n_vertices > 0) {
        OB_REQUIRE(u0 != nullptr, "ob_seed: null u0");
        OB_CUDA(cudaMemsetAsync(u0, 0, sizeof(double) * (size_t)n_vertices, stream));
    }
    if (n_sources == 0) return OB_OK;
    OB_REQUIRE(sources != nullptr, "ob_seed: null sources");
    seed_kernel<<<ceil_div(n_sources, kThreads), kThreads, 0, stream>>>(sources, n_sources,
                                                                        n_vertices, u0, invalid);
    OB_CHECK_LAUNCH("seed");
    return OB_OK;
}

int ob_grad_div(const float* xyz, const int32_t* faces, int n_faces, int n_vertices,
                const float* normals, const float* areas, const double* u, const float* cot,
                int n_columns, double* neg_div, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 0 && n_vertices >= 0 && n_columns >= 1, "ob_grad_div: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(neg_div != nullptr, "ob_grad_div: null output");
    OB_CUDA(cudaMemsetAsync(neg_div, 0, sizeof(double) * (size_t)n_vertices * n_columns, stream));
    if (n_faces == 0) return OB_OK;
    OB_REQUIRE(xyz && faces && normals && areas && u && cot, "ob_grad_div: null pointer");
    const long long total = (long long)n_faces * n_columns;
    grad_div_kernel<<<ceil_div(total, kThreads), kThreads, 0, stream>>>(
        xyz, faces, n_faces, normals, areas, u, cot, n_columns, neg_div);
    OB_CHECK_LAUNCH("grad_div");
    return OB_OK;
}

int ob_shift(double* phi, int n_vertices, const int32_t* sources, int n_sources,
             const int32_t* source_offsets, int n_columns, int orient, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && n_columns >= 1 && n_sources >= 0, "ob_shift: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(phi != nullptr && sources != nullptr, "ob_shift: null pointer");
    OB_REQUIRE(n_columns == 1 || source_offsets != nullptr,
               "ob_shift: several columns need source_offsets");
    OB_REQUIRE(source_offsets != nullptr || n_sources > 0, "ob_shift: no sources");
    const int blocks = std::max(1, std::min(ceil_div(n_vertices, kThreads * 4), 2 * sm_count()));
    Scratch scratch(stream);
    double2* partials = scratch.take<double2>((size_t)blocks * n_columns);
    double2* sums = scratch.take<double2>(n_columns);
    unsigned int* counter = scratch.take<unsigned int>(1);
    int st = scratch.commit();
    if (st) return st;
    OB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned int), stream));
    source_sums_kernel<<<dim3(blocks, n_columns), kThreads, 0, stream>>>(
        phi, n_vertices, sources, source_offsets, n_sources, n_columns, partials, counter, sums);
    OB_CHECK_LAUNCH("source_sums");
    const long long total = (long long)n_vertices * n_columns;
    shift_kernel<<<ceil_div(total, kThreads), kThreads, 0, stream>>>(
        phi, n_vertices, sums, source_offsets, n_sources, n_columns, orient);
    OB_CHECK_LAUNCH("shift");
    return OB_OK;
}

}  // extern "C"
