// a2-a5: per-face terms, the default time step's edge sums and the three operators' rows.
#include <cstring>

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
// (shift_factor, shifted_scalar_entry).
// Row i of L, H = factor L + M and P = -L (and its mass), the one arithmetic of both kernels below:
// each off-diagonal entry the sum of its run's half-cotangents in sorted order, the diagonal minus
// the row's off-diagonal sum in entry order. A group of kRowLanes lanes takes a row (entries
// base + lane, base + lane + kRowLanes, ...), so its columns, run starts and L/H/P entries are read
// and written as one contiguous run per group, where a thread a row would touch a line per entry;
// every lane of the group folds each chunk's off-diagonal values in entry order through shuffles.
constexpr int kRowLanes = 8;

template <typename C>
__device__ __forceinline__ void heat_row_lanes(int i, const int* __restrict__ offsets, const int* __restrict__ columns,
                                               const int* __restrict__ run_start,
                                               const unsigned long long* __restrict__ keys, int count,
                                               const int* __restrict__ order, const C* __restrict__ cot,
                                               double factor, const double* __restrict__ area_sums,
                                               double mass_divisor, double* __restrict__ L, double* __restrict__ H,
                                               double* __restrict__ P, double* __restrict__ mass) {
    const int lane = threadIdx.x % kRowLanes;
    const unsigned group = 0xFFu << (threadIdx.x & 31 & ~(kRowLanes - 1));
    const double m = area_sums[i] / mass_divisor;
    if (lane == 0) mass[i] = m;
    const int start = offsets[i], end = offsets[i + 1];
    double total = 0.0;
    int slot = -1;
    for (int base = start; base < end; base += kRowLanes) {
        const int k = base + lane;
        double value = 0.0;
        int off = 0;
        if (k < end) {
            if (columns[k] == i) {
                slot = k;
            } else {
                const int s = run_start[k];
                const int e = run_end(keys, s, count);
                for (int p = s; p < e; ++p) value += (double)cot[order[p]];
                L[k] = value;
                H[k] = factor * value;
                P[k] = -value;
                off = 1;
            }
        }
#pragma unroll
        for (int j = 0; j < kRowLanes; ++j) {
            const double v = __shfl_sync(group, value, j, kRowLanes);
            if (__shfl_sync(group, off, j, kRowLanes)) total += v;
        }
    }
    if (slot >= 0) {
        const double diagonal = -total;
        L[slot] = diagonal;
        H[slot] = __dmul_rn(factor, diagonal) + m;
        P[slot] = -diagonal;
    }
}

// The half-cotangent table is float32 (the extrinsic path, as the reference's) or float64 (the
// intrinsic cover's, formed from float64 lengths: kernels/heat.py:1133, HEAT_SYSTEM_ROWS[float64]).
template <typename C>
__global__ void heat_rows_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                                 const int* __restrict__ run_start,
                                 const unsigned long long* __restrict__ keys, int count,
                                 const int* __restrict__ order, int n, const C* __restrict__ cot,
                                 double scale, const double* __restrict__ edge_sums, int from_edges,
                                 const double* __restrict__ area_sums, double mass_divisor,
                                 double* __restrict__ L, double* __restrict__ H,
                                 double* __restrict__ P, double* __restrict__ mass) {
    const int i = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) / kRowLanes);
    if (i >= n) return;
    double factor = scale;
    if (from_edges) {
        double h = 0.0;
        if (edge_sums[1] > 0.0) h = edge_sums[0] / edge_sums[1];
        factor = scale * (h * h);
    }
    heat_row_lanes(i, offsets, columns, run_start, keys, count, order, cot, factor, area_sums, mass_divisor,
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
    const int i = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) / kRowLanes);
    if (i >= n) return;
    heat_row_lanes(i, offsets, columns, run_start, keys, count, order, cot, row_factor[i], area_sums,
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

// ordito/kernels/triangles.py:276-330 (face_voronoi_areas): Meyer et al.'s mixed areas per
// corner, formed in float64 from the float32 corners and rounded once to float32 -- a non-obtuse
// face splits by its circumcentre weights, an obtuse one gives half its area to the obtuse
// corner and a quarter to each other, a degenerate one splits evenly -- and each share added
// exactly (float64 of the float32) into its corner's sum (kernels/heat.py:128-131).
__global__ void voronoi_area_sums_kernel(const float* __restrict__ xyz, const int* __restrict__ faces,
                                         int n_faces, double* __restrict__ area_sums) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const int i0 = faces[3 * f], i1 = faces[3 * f + 1], i2 = faces[3 * f + 2];
    const f3 a = load_f3(xyz, i0), b = load_f3(xyz, i1), c = load_f3(xyz, i2);
    const double p0x = a.x, p0y = a.y, p0z = a.z, p1x = b.x, p1y = b.y, p1z = b.z;
    const double p2x = c.x, p2y = c.y, p2z = c.z;
    auto length = [](double x, double y, double z) { return sqrt(x * x + y * y + z * z); };
    const double l0 = length(p1x - p2x, p1y - p2y, p1z - p2z);
    const double l1 = length(p2x - p0x, p2y - p0y, p2z - p0z);
    const double l2 = length(p0x - p1x, p0y - p1y, p0z - p1z);
    const double ex = p1x - p0x, ey = p1y - p0y, ez = p1z - p0z;
    const double fx = p2x - p0x, fy = p2y - p0y, fz = p2z - p0z;
    const double area = 0.5 * length(ey * fz - ez * fy, ez * fx - ex * fz, ex * fy - ey * fx);
    const double even = area / 3.0;
    double q0 = even, q1 = even, q2 = even;
    if (l0 > 0.0 && l1 > 0.0 && l2 > 0.0) {
        const double c0 = (l2 * l2 + l1 * l1 - l0 * l0) / (2.0 * l1 * l2);
        const double c1 = (l0 * l0 + l2 * l2 - l1 * l1) / (2.0 * l2 * l0);
        const double c2 = (l1 * l1 + l0 * l0 - l2 * l2) / (2.0 * l0 * l1);
        const double b0 = c0 * l0, b1 = c1 * l1, b2 = c2 * l2;
        const double weight = b0 + b1 + b2;
        if (weight != 0.0) {
            const double partial0 = b0 / weight * area, partial1 = b1 / weight * area;
            const double partial2 = b2 / weight * area;
            q0 = 0.5 * (partial1 + partial2);
            q1 = 0.5 * (partial2 + partial0);
            q2 = 0.5 * (partial0 + partial1);
        }
        const double half = 0.5 * area, quarter = 0.25 * area;
        if (c0 < 0.0) {
            q0 = half;
            q1 = quarter;
            q2 = quarter;
        } else if (c1 < 0.0) {
            q0 = quarter;
            q1 = half;
            q2 = quarter;
        } else if (c2 < 0.0) {
            q0 = quarter;
            q1 = quarter;
            q2 = half;
        }
    }
    atomicAdd(&area_sums[i0], (double)(float)q0);
    atomicAdd(&area_sums[i1], (double)(float)q1);
    atomicAdd(&area_sums[i2], (double)(float)q2);
}

// ordito/kernels/heat.py:469-485 (rim_vertices) with kernels/laplacian.py:1286-1321
// (pattern_row_on_rim): a vertex is on the rim when one of its off-diagonal entries' runs holds a
// single corner key (that edge lies on one face); their count is added to *n_rim.
__global__ void rim_vertices_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                                    const int* __restrict__ run_start, const unsigned long long* __restrict__ keys,
                                    int count, int n, int* __restrict__ rim, int* __restrict__ n_rim) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int on_rim = 0;
    for (int k = offsets[i]; k < offsets[i + 1] && !on_rim; ++k)
        if (columns[k] != i && run_end(keys, run_start[k], count) - run_start[k] == 1) on_rim = 1;
    rim[i] = on_rim;
    if (on_rim) atomicAdd(n_rim, 1);
}

// ordito/kernels/heat.py:488-509 (pinned_heat_rows): the heat system with the solution pinned to
// zero on the rim -- a rim row becomes the identity's, an interior row drops its rim columns.
__global__ void pinned_rows_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                                   const int* __restrict__ rim, const double* __restrict__ values, int n,
                                   double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = offsets[i]; k < offsets[i + 1]; ++k) {
        const int c = columns[k];
        double v = values[k];
        if (rim[i] != 0)
            v = (c == i) ? 1.0 : 0.0;
        else if (rim[c] != 0)
            v = 0.0;
        out[k] = v;
    }
}

// kernels/heat.py:512-515 (off_rim): the pinned solve's right-hand side, zero on the rim.
__global__ void off_rim_kernel(const double* __restrict__ in, const int* __restrict__ rim, int n,
                               double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = rim[i] != 0 ? 0.0 : in[i];
}

// ordito/heat.py:4098-4114 (add_to_diagonal): values + shift on the diagonal entries.
__global__ void add_to_diagonal_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                                       const double* __restrict__ values, int n, double shift,
                                       double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = offsets[i]; k < offsets[i + 1]; ++k) out[k] = values[k] + (columns[k] == i ? shift : 0.0);
}

// ordito/laplacian.py:779-874 (mollify_intrinsic), kernels/laplacian.py:1585-1627
// (face_edge_lengths_and_margin): each face's float32 side lengths, column e opposite corner e
// (kernels/predicates.py:221), and the smallest triangle-inequality margin a + b - c over every
// face and side (*margin, an order-preserving int encoding of a float, seeded +inf), with the
// lengths' float64 sum (*total) for their mean.
__device__ __forceinline__ int ordered_bits(float x) {
    const int i = __float_as_int(x);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
inline float from_ordered_bits(int i) {
    const int bits = i >= 0 ? i : i ^ 0x7fffffff;
    float x;
    std::memcpy(&x, &bits, sizeof(float));
    return x;
}

__global__ void face_lengths_margin_kernel(const float* __restrict__ xyz, const int* __restrict__ faces,
                                           int n_faces, float* __restrict__ lengths, int* __restrict__ margin,
                                           double* __restrict__ total) {
    __shared__ float low[kThreads / 32];
    __shared__ double sum[kThreads / 32];
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    float m = INFINITY;
    double s = 0.0;
    if (f < n_faces) {
        const f3 v0 = load_f3(xyz, faces[3 * f]), v1 = load_f3(xyz, faces[3 * f + 1]);
        const f3 v2 = load_f3(xyz, faces[3 * f + 2]);
        auto length = [](float x, float y, float z) { return sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z))); };
        const float a = length(v1.x - v2.x, v1.y - v2.y, v1.z - v2.z);
        const float b = length(v2.x - v0.x, v2.y - v0.y, v2.z - v0.z);
        const float c = length(v0.x - v1.x, v0.y - v1.y, v0.z - v1.z);
        lengths[3 * f] = a;
        lengths[3 * f + 1] = b;
        lengths[3 * f + 2] = c;
        m = fminf(fminf(a + b - c, b + c - a), c + a - b);
        s = (double)a + (double)b + (double)c;
    }
    for (int o = 16; o > 0; o >>= 1) {
        m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
        s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    if ((threadIdx.x & 31) == 0) {
        low[threadIdx.x / 32] = m;
        sum[threadIdx.x / 32] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float bm = INFINITY;
        double bs = 0.0;
        for (int w = 0; w < (int)blockDim.x / 32; ++w) {
            bm = fminf(bm, low[w]);
            bs += sum[w];
        }
        atomicMin(margin, ordered_bits(bm));
        atomicAdd(total, bs);
    }
}

// ordito/kernels/laplacian.py:56-90 (cot_entries_from_l2, cot_entries_from_edge_lengths) and
// kernels/predicates.py:194-210 (doublearea_from_lengths, Kahan's Heron with the largest side
// first): the float32 half-cotangents of a face from its lengths plus delta.
__global__ void intrinsic_cot_kernel(const float* __restrict__ lengths, int n_faces, float delta,
                                     float* __restrict__ cot) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const float l0 = __fadd_rn(lengths[3 * f], delta), l1 = __fadd_rn(lengths[3 * f + 1], delta);
    const float l2 = __fadd_rn(lengths[3 * f + 2], delta);
    // Sorted ascending (c <= b <= a): the largest side first in Kahan's product.
    float c = l0, b = l1, a = l2, t;
    if (c > b) t = c, c = b, b = t;
    if (b > a) t = b, b = a, a = t;
    if (c > b) t = c, c = b, b = t;
    const float arg = __fmul_rn(__fmul_rn(__fmul_rn(__fadd_rn(a, __fadd_rn(b, c)), __fsub_rn(c, __fsub_rn(a, b))),
                                          __fadd_rn(c, __fsub_rn(a, b))),
                                __fadd_rn(a, __fsub_rn(b, c)));
    float dbl_area = __fmul_rn(0.5f, sqrtf(fmaxf(arg, 0.0f)));
    if (isnan(dbl_area)) dbl_area = 0.0f;
    const float denominator = __fmul_rn(4.0f, dbl_area);
    float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
    if (denominator > 0.0f) {
        const float s0 = __fmul_rn(l0, l0), s1 = __fmul_rn(l1, l1), s2 = __fmul_rn(l2, l2);
        c0 = __fdiv_rn(__fsub_rn(__fadd_rn(s1, s2), s0), denominator);
        c1 = __fdiv_rn(__fsub_rn(__fadd_rn(s2, s0), s1), denominator);
        c2 = __fdiv_rn(__fsub_rn(__fadd_rn(s0, s1), s2), denominator);
    }
    cot[3 * f] = c0;
    cot[3 * f + 1] = c1;
    cot[3 * f + 2] = c2;
}

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_mollified_cot(const float* xyz, const int32_t* faces, int n_faces, double epsilon, float* lengths,
                     float* cot, double* delta_out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 0 && delta_out != nullptr, "ob_mollified_cot: bad argument");
    *delta_out = 0.0;
    if (n_faces == 0) return OB_OK;
    OB_REQUIRE(xyz && faces && lengths && cot, "ob_mollified_cot: null pointer");
    Scratch scratch(stream);
    int* margin = scratch.take<int>(1);
    double* total = scratch.take<double>(1);
    int st = scratch.commit();
    if (st) return st;
    const int inf_bits = 0x7f800000;  // +inf, whose ordered encoding is its own bits
    OB_CUDA(cudaMemcpyAsync(margin, &inf_bits, sizeof(int), cudaMemcpyHostToDevice, stream));
    OB_CUDA(cudaMemsetAsync(total, 0, sizeof(double), stream));
    face_lengths_margin_kernel<<<ceil_div(n_faces, kThreads), kThreads, 0, stream>>>(xyz, faces, n_faces, lengths,
                                                                                   margin, total);
    OB_CHECK_LAUNCH("face_lengths_margin");
    int margin_bits = 0;
    double sum = 0.0;
    OB_CUDA(cudaMemcpyAsync(&margin_bits, margin, sizeof(int), cudaMemcpyDeviceToHost, stream));
    OB_CUDA(cudaMemcpyAsync(&sum, total, sizeof(double), cudaMemcpyDeviceToHost, stream));
    OB_CUDA(cudaStreamSynchronize(stream));
    // delta = max(epsilon * mean length - margin, 0) in float32 (laplacian.py:864-867).
    const float epsilon_scaled = (float)(epsilon * (sum / (3.0 * (double)n_faces)));
    const float delta = std::max(epsilon_scaled - from_ordered_bits(margin_bits), 0.0f);
    intrinsic_cot_kernel<<<ceil_div(n_faces, kThreads), kThreads, 0, stream>>>(lengths, n_faces, delta, cot);
    OB_CHECK_LAUNCH("intrinsic_cot");
    *delta_out = (double)delta;
    return OB_OK;
}

int ob_voronoi_area_sums(const float* xyz, const int32_t* faces, int n_faces, int n_vertices,
                         double* area_sums, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 0 && n_vertices >= 0, "ob_voronoi_area_sums: negative size");
    if (n_vertices > 0) {
        OB_REQUIRE(area_sums != nullptr, "ob_voronoi_area_sums: null area_sums");
        OB_CUDA(cudaMemsetAsync(area_sums, 0, sizeof(double) * (size_t)n_vertices, stream));
    }
    if (n_faces == 0) return OB_OK;
    OB_REQUIRE(xyz && faces, "ob_voronoi_area_sums: null pointer");
    voronoi_area_sums_kernel<<<ceil_div(n_faces, kThreads), kThreads, 0, stream>>>(xyz, faces, n_faces,
                                                                                   area_sums);
    OB_CHECK_LAUNCH("voronoi_area_sums");
    return OB_OK;
}

int ob_rim_vertices(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                    const uint64_t* keys, int count, int n_vertices, int32_t* rim, int32_t* n_rim,
                    ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && n_rim != nullptr, "ob_rim_vertices: bad argument");
    OB_CUDA(cudaMemsetAsync(n_rim, 0, sizeof(int32_t), stream));
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(offsets && columns && run_start && keys && rim, "ob_rim_vertices: null pointer");
    rim_vertices_kernel<<<ceil_div(n_vertices, kThreads), kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), count, n_vertices, rim,
        n_rim);
    OB_CHECK_LAUNCH("rim_vertices");
    return OB_OK;
}

int ob_pinned_rows(const int32_t* offsets, const int32_t* columns, const int32_t* rim, const double* values,
                   int n_vertices, double* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0, "ob_pinned_rows: negative size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(offsets && columns && rim && values && out, "ob_pinned_rows: null pointer");
    pinned_rows_kernel<<<ceil_div(n_vertices, kThreads), kThreads, 0, stream>>>(offsets, columns, rim, values,
                                                                                 n_vertices, out);
    OB_CHECK_LAUNCH("pinned_rows");
    return OB_OK;
}

int ob_off_rim(const double* in, const int32_t* rim, int n_vertices, double* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0, "ob_off_rim: negative size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(in && rim && out, "ob_off_rim: null pointer");
    off_rim_kernel<<<ceil_div(n_vertices, kThreads), kThreads, 0, stream>>>(in, rim, n_vertices, out);
    OB_CHECK_LAUNCH("off_rim");
    return OB_OK;
}

int ob_add_to_diagonal(const int32_t* offsets, const int32_t* columns, const double* values, int n_vertices,
                       double shift, double* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0, "ob_add_to_diagonal: negative size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(offsets && columns && values && out, "ob_add_to_diagonal: null pointer");
    add_to_diagonal_kernel<<<ceil_div(n_vertices, kThreads), kThreads, 0, stream>>>(offsets, columns, values,
                                                                                     n_vertices, shift, out);
    OB_CHECK_LAUNCH("add_to_diagonal");
    return OB_OK;
}

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
    heat_rows_packed_kernel<<<ceil_div((long long)n_vertices * kRowLanes, kThreads), kThreads, 0, stream>>>(
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
    heat_rows_kernel<float><<<ceil_div((long long)n_vertices * kRowLanes, kThreads), kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), count,
        order, n_vertices, cot, scale, edge_sums, from_edges, area_sums, mass_divisor, L, H, P,
        mass);
    OB_CHECK_LAUNCH("heat_rows");
    return OB_OK;
}

int ob_heat_rows_f64(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                     const uint64_t* keys, int count, const int32_t* order, int n_vertices,
                     const double* cot, double scale, const double* edge_sums, int from_edges,
                     const double* area_sums, double mass_divisor, double* L, double* H, double* P,
                     double* mass, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    if (n_vertices <= 0) return OB_OK;
    OB_REQUIRE(offsets && columns && run_start && keys && order && cot && area_sums && L && H &&
                   P && mass,
               "ob_heat_rows_f64: null pointer");
    OB_REQUIRE(!from_edges || edge_sums != nullptr, "ob_heat_rows_f64: from_edges needs edge_sums");
    heat_rows_kernel<double><<<ceil_div((long long)n_vertices * kRowLanes, kThreads), kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), count,
        order, n_vertices, cot, scale, edge_sums, from_edges, area_sums, mass_divisor, L, H, P,
        mass);
    OB_CHECK_LAUNCH("heat_rows_f64");
    return OB_OK;
}

}  // extern "C"
