// a2-a5: per-face terms, the default time step's edge sums and the three operators' rows.
#include "ob_geometry.cuh"
#include "ob_internal.cuh"
#include "ob_scratch.cuh"

namespace ob {
namespace {

constexpr int kThreads = 256;

// ordito/kernels/heat.py:92-131 (heat_face_terms, barycentric mass): one thread per face writes
// its half-cotangents, unit normal and area, and adds the area exactly (float64 of a float32)
// into each corner's sum.
__global__ void face_terms_kernel(const float* __restrict__ xyz, const int* __restrict__ faces,
                                  int n_faces, int n, float* __restrict__ cot,
                                  float* __restrict__ normals, float* __restrict__ areas,
                                  double* __restrict__ area_sums) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const int i0 = faces[3 * f], i1 = faces[3 * f + 1], i2 = faces[3 * f + 2];
    const f3 v0 = load_f3(xyz, i0), v1 = load_f3(xyz, i1), v2 = load_f3(xyz, i2);
    if (cot != nullptr) {
        float c[3];
        half_cotangents(v0, v1, v2, c);
        cot[3 * f] = c[0];
        cot[3 * f + 1] = c[1];
        cot[3 * f + 2] = c[2];
    }
    f3 nrm;
    float area;
    normal_and_area(v0, v1, v2, &nrm, &area);
    normals[3 * f] = nrm.x;
    normals[3 * f + 1] = nrm.y;
    normals[3 * f + 2] = nrm.z;
    areas[f] = area;
    const double a = (double)area;
    atomicAdd(&area_sums[i0], a);
    atomicAdd(&area_sums[i1], a);
    atomicAdd(&area_sums[i2], a);
}

__device__ __forceinline__ int run_end(const unsigned long long* __restrict__ keys, int start,
                                       int count) {
    const unsigned long long key = keys[start];
    int p = start + 1;
    while (p < count && keys[p] == key) ++p;
    return p;
}

// ordito/kernels/heat.py:143-237 (upper_edge_length_sum_and_count): a grid-stride walk over rows,
// one fixed-tree block sum per quantity, folded in block order by the last block to finish.
__global__ void edge_sums_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                                 const int* __restrict__ run_start,
                                 const unsigned long long* __restrict__ keys, int count, int n,
                                 const float* __restrict__ xyz, int face_edges,
                                 double2* __restrict__ partials, unsigned int* counter,
                                 double* __restrict__ out) {
    __shared__ double scratch[32];
    __shared__ int last;
    double sum = 0.0, cnt = 0.0;
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        const f3 vr = load_f3(xyz, row);
        for (int k = offsets[row]; k < offsets[row + 1]; ++k) {
            const int col = columns[k];
            if (col <= row) continue;
            double weight = 1.0;
            if (face_edges) {
                const int s = run_start[k];
                weight = (double)(run_end(keys, s, count) - s);
            }
            sum += weight * (double)length(sub(load_f3(xyz, col), vr));
            cnt += weight;
        }
    }
    const double bs = block_sum(sum, scratch);
    const double bc = block_sum(cnt, scratch);
    if (threadIdx.x == 0) partials[blockIdx.x] = make_double2(bs, bc);
    if (!last_block_arrived(counter, &last)) return;
    if (threadIdx.x == 0) {
        double s = 0.0, c = 0.0;
        for (int b = 0; b < (int)gridDim.x; ++b) {
            const double2 p = __ldcg(&partials[b]);
            s += p.x;
            c += p.y;
        }
        out[0] = s;
        out[1] = c;
    }
}

// ordito/kernels/heat.py:299-465 (heat_system_rows, scalar_heat_row, scalar_heat_diagonal),
// kernels/laplacian.py:971-989 (cotmatrix_offdiagonal), kernels/linalg.py:1594-1621
// (shift_factor, shifted_scalar_entry): one thread per row walks its entries in row order.
// Row i of L, H = factor L + M and P = -L (and its mass), the one arithmetic of both kernels below.
__device__ __forceinline__ void heat_row(int i, const int* __restrict__ offsets, const int* __restrict__ columns,
                                         const int* __restrict__ run_start,
                                         const unsigned long long* __restrict__ keys, int count,
                                         const int* __restrict__ order, const float* __restrict__ cot,
                                         double factor, const double* __restrict__ area_sums,
                                         double mass_divisor, double* __restrict__ L, double* __restrict__ H,
                                         double* __restrict__ P, double* __restrict__ mass) {
    const double m = area_sums[i] / mass_divisor;
    mass[i] = m;
    const int start = offsets[i], end = offsets[i + 1];
    double total = 0.0;
    int slot = -1;
    for (int k = start; k < end; ++k) {
        if (columns[k] == i) {
            slot = k;
            continue;
        }
        const int s = run_start[k];
        const int e = run_end(keys, s, count);
        double value = 0.0;
        for (int p = s; p < e; ++p) value += (double)cot[order[p]];
        L[k] = value;
        total += value;
        H[k] = factor * value;
        P[k] = -value;
    }
    if (slot >= 0) {
        const double diagonal = -total;
        L[slot] = diagonal;
        H[slot] = __dmul_rn(factor, diagonal) + m;
        P[slot] = -diagonal;
    }
}

__global__ void heat_rows_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                                 const int* __restrict__ run_start,
                                 const unsigned long long* __restrict__ keys, int count,
                                 const int* __restrict__ order, int n, const float* __restrict__ cot,
                                 double scale, const double* __restrict__ edge_sums, int from_edges,
                                 const double* __restrict__ area_sums, double mass_divisor,
                                 double* __restrict__ L, double* __restrict__ H,
                                 double* __restrict__ P, double* __restrict__ mass) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double factor = scale;
    if (from_edges) {
        double h = 0.0;
        if (edge_sums[1] > 0.0) h = edge_sums[0] / edge_sums[1];
        factor = scale * (h * h);
    }
    heat_row(i, offsets, columns, run_start, keys, count, order, cot, factor, area_sums, mass_divisor,
             L, H, P, mass);
}

// Many meshes packed as one block-diagonal operator: each row's own factor (its mesh's -t).
__global__ void heat_rows_packed_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                                        const int* __restrict__ run_start,
                                        const unsigned long long* __restrict__ keys, int count,
                                        const int* __restrict__ order, int n, const float* __restrict__ cot,
                                        const double* __restrict__ row_factor,
                                        const double* __restrict__ area_sums, double mass_divisor,
                                        double* __restrict__ L, double* __restrict__ H,
                                        double* __restrict__ P, double* __restrict__ mass) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    heat_row(i, offsets, columns, run_start, keys, count, order, cot, row_factor[i], area_sums,
             mass_divisor, L, H, P, mass);
}

// Per segment of rows (a packed mesh): edge_sums_kernel's two sums over its strict upper
// triangle, one block a segment, added in a fixed order.
__global__ void edge_sums_segments_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                                          const int* __restrict__ run_start,
                                          const unsigned long long* __restrict__ keys, int count,
                                          const float* __restrict__ xyz, int face_edges,
                                          const int* __restrict__ segments, double* __restrict__ out) {
    __shared__ double scratch[32];
    const int s = blockIdx.x;
    double sum = 0.0, cnt = 0.0;
    for (int row = segments[s] + threadIdx.x; row < segments[s + 1]; row += blockDim.x) {
        const f3 vr = load_f3(xyz, row);
        for (int k = offsets[row]; k < offsets[row + 1]; ++k) {
            const int col = columns[k];
            if (col <= row) continue;
            double weight = 1.0;
            if (face_edges) {
                const int r = run_start[k];
                weight = (double)(run_end(keys, r, count) - r);
            }
            sum += weight * (double)length(sub(load_f3(xyz, col), vr));
            cnt += weight;
        }
    }
    const double bs = block_sum(sum, scratch);
    const double bc = block_sum(cnt, scratch);
    if (threadIdx.x == 0) {
        out[2 * s] = bs;
        out[2 * s + 1] = bc;
    }
}

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_face_terms(const float* xyz, const int32_t* faces, int n_faces, int n_vertices, float* cot,
                  float* normals, float* areas, double* area_sums, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 0 && n_vertices >= 0, "ob_face_terms: negative size");
    if (n_vertices > 0) {
        OB_REQUIRE(area_sums != nullptr, "ob_face_terms: null area_sums");
        OB_CUDA(cudaMemsetAsync(area_sums, 0, sizeof(double) * (size_t)n_vertices, stream));
    }
    if (n_faces == 0) return OB_OK;
    OB_REQUIRE(xyz && faces && normals && areas, "ob_face_terms: null pointer");
    face_terms_kernel<<<ceil_div(n_faces, kThreads), kThreads, 0, stream>>>(
        xyz, faces, n_faces, n_vertices, cot, normals, areas, area_sums);
    OB_CHECK_LAUNCH("face_terms");
    return OB_OK;
}

int ob_edge_sums(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                 const uint64_t* keys, int count, int n_vertices, const float* xyz,
                 int face_edges, double* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(out != nullptr, "ob_edge_sums: null output");
    if (n_vertices <= 0) {
        OB_CUDA(cudaMemsetAsync(out, 0, 2 * sizeof(double), stream));
        return OB_OK;
    }
    OB_REQUIRE(offsets && columns && run_start && keys && xyz, "ob_edge_sums: null pointer");
    const int blocks = std::min(ceil_div(n_vertices, kThreads), 4 * sm_count());
    Scratch scratch(stream);
    double2* partials = scratch.take<double2>(blocks);
    unsigned int* counter = scratch.take<unsigned int>(1);
    int st = scratch.commit();
    if (st) return st;
    OB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned int), stream));
    edge_sums_kernel<<<blocks, kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), count,
        n_vertices, xyz, face_edges, partials, counter, out);
    OB_CHECK_LAUNCH("edge_sums");
    return OB_OK;
}

int ob_edge_sums_segments(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                          const uint64_t* keys, int count, const float* xyz, int face_edges,
                          const int32_t* segments, int n_segments, double* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_segments >= 0 && out, "ob_edge_sums_segments: bad argument");
    if (n_segments == 0) return OB_OK;
    OB_REQUIRE(offsets && columns && run_start && keys && xyz && segments, "ob_edge_sums_segments: null pointer");
    edge_sums_segments_kernel<<<n_segments, kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), count, xyz,
        face_edges, segments, out);
    OB_CHECK_LAUNCH("edge_sums_segments");
    return OB_OK;
}

int ob_heat_rows_packed(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                        const uint64_t* keys, int count, const int32_t* order, int n_vertices,
                        const float* cot, const double* row_factor, const double* area_sums,
                        double mass_divisor, double* L, double* H, double* P, double* mass,
                        ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    if (n_vertices <= 0) return OB_OK;
    OB_REQUIRE(offsets && columns && run_start && keys && order && cot && row_factor && area_sums && L &&
                   H && P && mass,
               "ob_heat_rows_packed: null pointer");
    heat_rows_packed_kernel<<<ceil_div(n_vertices, kThreads), kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), count, order,
        n_vertices, cot, row_factor, area_sums, mass_divisor, L, H, P, mass);
    OB_CHECK_LAUNCH("heat_rows_packed");
    return OB_OK;
}

int ob_heat_rows(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                 const uint64_t* keys, int count, const int32_t* order, int n_vertices,
                 const float* cot, double scale, const double* edge_sums, int from_edges,
                 const double* area_sums, double mass_divisor, double* L, double* H, double* P,
                 double* mass, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    if (n_vertices <= 0) return OB_OK;
    OB_REQUIRE(offsets && columns && run_start && keys && order && cot && area_sums && L && H &&
                   P && mass,
               "ob_heat_rows: null pointer");
    OB_REQUIRE(!from_edges || edge_sums != nullptr, "ob_heat_rows: from_edges needs edge_sums");
    heat_rows_kernel<<<ceil_div(n_vertices, kThreads), kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), count,
        order, n_vertices, cot, scale, edge_sums, from_edges, area_sums, mass_divisor, L, H, P,
        mass);
    OB_CHECK_LAUNCH("heat_rows");
    return OB_OK;
}

}  // extern "C"
