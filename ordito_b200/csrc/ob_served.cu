// The served batch's per-query kernels, atomic-free and in the factors' own numbering.
//
// A served batch solves k right-hand sides against two held Cholesky factors that share one
// ordering (the Poisson factor reuses the heat factor's analysis). These kernels let the batch
// stay in that ordering between the two solves: the seeds are written straight into the heat
// factor's right-hand side, the divergence reads the heat solution and writes the Poisson
// right-hand side through the ordering's inverse permutation, and the shift reads the Poisson
// solution the same way while writing the (k, V) distances out -- no permutation or transpose
// passes between them.
//
// The divergence is gathered per vertex rather than scattered per face (ordito/kernels/heat.py:
// 626-687 accumulates with float64 atomics, or under its deterministic mode stores per corner
// and sums each vertex's corners in ascending corner order, ordito/heat.py:3170-3232): each
// (vertex, column) thread walks the vertex's corners in ascending slot order (a stable sort of
// the face buffer by vertex, ordito/heat.py:3198 _corner_order) and recomputes each incident
// face's unit gradient itself. No atomics, the same bits on every run, and no per-corner table.
#include <cub/device/device_radix_sort.cuh>

#include "ob_geometry.cuh"
#include "ob_internal.cuh"
#include "ob_scratch.cuh"

namespace ob {
namespace {

constexpr int kThreads = 256;

__global__ void corner_keys_kernel(const int* __restrict__ faces, int n_corners, int n,
                                   int* __restrict__ keys, int* __restrict__ slots) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_corners) return;
    const int v = faces[q];
    keys[q] = (v >= 0 && v < n) ? v : n;
    slots[q] = q;
}

// offsets[v] = first sorted position of vertex v (every vertex, empty ones included).
__global__ void corner_offsets_kernel(const int* __restrict__ sorted, int n_corners, int n,
                                      int* __restrict__ offsets) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > n_corners) return;
    const int here = p < n_corners ? sorted[p] : n;
    const int before = p > 0 ? sorted[p - 1] : -1;
    for (int v = before + 1; v <= here && v <= n; ++v) offsets[v] = p;
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

// Row of vertex v in a buffer: its own index, or its position in the factor's ordering.
__device__ __forceinline__ int row_of(const int* __restrict__ iperm, int v) {
    return iperm ? iperm[v] : v;
}

// -div of the unit gradient at (vertex, column), summed over the vertex's corners in ascending
// slot order: the same arithmetic per face as ob_grad_div (kernels/triangles.py:834-894,
// kernels/predicates.py:719-724, kernels/heat.py:626-687), the corner's own term kept.
__global__ void grad_div_gather_kernel(const float* __restrict__ xyz, const int* __restrict__ faces,
                                       const float* __restrict__ normals,
                                       const float* __restrict__ areas,
                                       const float* __restrict__ cot,
                                       const int* __restrict__ corner_offsets,
                                       const int* __restrict__ corner_slots, int n, int k,
                                       const double* __restrict__ u, int u_stride,
                                       const int* __restrict__ u_iperm, double* __restrict__ out,
                                       int out_stride, const int* __restrict__ out_iperm,
                                       const char* __restrict__ out_pinned) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * out_stride) return;
    const int v = (int)(t / out_stride), c = (int)(t % out_stride);
    if (c >= k) {
        // A pad column of the output stays zero.
        out[(size_t)row_of(out_iperm, v) * out_stride + c] = 0.0;
        return;
    }
    double acc = 0.0;
    for (int p = corner_offsets[v]; p < corner_offsets[v + 1]; ++p) {
        const int q = corner_slots[p];
        const int f = q / 3, e = q - 3 * f;
        const int i0 = faces[3 * f], i1 = faces[3 * f + 1], i2 = faces[3 * f + 2];
        const d3 v0 = widen(load_f3(xyz, i0)), v1 = widen(load_f3(xyz, i1)),
                 v2 = widen(load_f3(xyz, i2));
        const d3 nrm = widen(load_f3(normals, f));
        const double area = (double)areas[f];
        // The unnormalised gradient sum_k u_k (n x e_k); its direction is the unit gradient's, and
        // the positive factor 1 / (2 A) cancels in the normalisation, so it is never divided in.
        d3 g{0.0, 0.0, 0.0};
        if (area > 0.0) {
            const double u0 = u[(size_t)row_of(u_iperm, i0) * u_stride + c];
            const double u1 = u[(size_t)row_of(u_iperm, i1) * u_stride + c];
            const double u2 = u[(size_t)row_of(u_iperm, i2) * u_stride + c];
            const d3 a = dcross(nrm, dsub(v2, v1)), b = dcross(nrm, dsub(v0, v2)),
                     w = dcross(nrm, dsub(v1, v0));
            g = d3{u0 * a.x + u1 * b.x + u2 * w.x, u0 * a.y + u1 * b.y + u2 * w.y,
                   u0 * a.z + u1 * b.z + u2 * w.z};
        }
        // Scaled by its largest component first so a far-field gradient's square cannot underflow
        // (kernels/predicates.py:719 stable_normalize), then one reciprocal square root.
        const double largest = fmax(fabs(g.x), fmax(fabs(g.y), fabs(g.z)));
        d3 x{0.0, 0.0, 0.0};
        if (largest != 0.0) {
            // A subnormal largest component would overflow its reciprocal: divide instead.
            d3 s;
            if (largest > 1e-300) {
                const double scale = 1.0 / largest;
                s = d3{g.x * scale, g.y * scale, g.z * scale};
            } else {
                s = d3{g.x / largest, g.y / largest, g.z / largest};
            }
            const double inv_len = rsqrt(ddot(s, s));
            x = d3{s.x * inv_len, s.y * inv_len, s.z * inv_len};
        }
        const double c0 = (double)cot[3 * f], c1 = (double)cot[3 * f + 1], c2 = (double)cot[3 * f + 2];
        double d;
        if (e == 0)
            d = c2 * ddot(dsub(v1, v0), x) + c1 * ddot(dsub(v2, v0), x);
        else if (e == 1)
            d = c0 * ddot(dsub(v2, v1), x) + c2 * ddot(dsub(v0, v1), x);
        else
            d = c1 * ddot(dsub(v0, v2), x) + c0 * ddot(dsub(v1, v2), x);
        acc += d;
    }
    const int row = row_of(out_iperm, v);
    out[(size_t)row * out_stride + c] = (out_pinned && out_pinned[row]) ? 0.0 : acc;
}

// out[i] = map[indices[i]]: a face buffer renumbered into a factor's ordering (grid-stride).
__global__ void renumber_kernel(const int* __restrict__ indices, long long count,
                                const int* __restrict__ map, int* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = map[indices[i]];
}

// Per-face terms of the divergence that do not depend on u (once per mesh), 18 doubles a face:
// the gradient bases n x e_k (e_0 = v2 - v1, e_1 = v0 - v2, e_2 = v1 - v0; zero for a face of
// no area, whose gradient is zero) and, per corner e, the cotangent-weighted edge sum W_e with
// d_e = W_e . X: W_0 = c2 (v1 - v0) + c1 (v2 - v0), W_1 = c0 (v2 - v1) + c2 (v0 - v1),
// W_2 = c1 (v0 - v2) + c0 (v1 - v2) (kernels/heat.py:626-687 forms the same d_e as two dots).
constexpr int kFaceTerms = 18;

__global__ void face_gradient_terms_kernel(const float* __restrict__ xyz, const int* __restrict__ faces,
                                           int n_faces, const float* __restrict__ normals,
                                           const float* __restrict__ areas, const float* __restrict__ cot,
                                           double* __restrict__ terms) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const d3 v0 = widen(load_f3(xyz, faces[3 * f])), v1 = widen(load_f3(xyz, faces[3 * f + 1])),
             v2 = widen(load_f3(xyz, faces[3 * f + 2]));
    const d3 nrm = widen(load_f3(normals, f));
    d3 a{0, 0, 0}, b{0, 0, 0}, w{0, 0, 0};
    if ((double)areas[f] > 0.0) {
        a = dcross(nrm, dsub(v2, v1));
        b = dcross(nrm, dsub(v0, v2));
        w = dcross(nrm, dsub(v1, v0));
    }
    const double c0 = (double)cot[3 * f], c1 = (double)cot[3 * f + 1], c2 = (double)cot[3 * f + 2];
    const d3 e10 = dsub(v1, v0), e20 = dsub(v2, v0), e21 = dsub(v2, v1);
    // W_1 = c0 (v2 - v1) + c2 (v0 - v1) = c0 e21 - c2 e10; W_2 = c1 (v0 - v2) + c0 (v1 - v2)
    // = -c1 e20 - c0 e21.
    const d3 W0{c2 * e10.x + c1 * e20.x, c2 * e10.y + c1 * e20.y, c2 * e10.z + c1 * e20.z};
    const d3 W1{c0 * e21.x - c2 * e10.x, c0 * e21.y - c2 * e10.y, c0 * e21.z - c2 * e10.z};
    const d3 W2{-c1 * e20.x - c0 * e21.x, -c1 * e20.y - c0 * e21.y, -c1 * e20.z - c0 * e21.z};
    double* T = terms + (size_t)kFaceTerms * f;
    const double values[kFaceTerms] = {a.x, a.y, a.z, b.x, b.y, b.z, w.x, w.y, w.z,
                                       W0.x, W0.y, W0.z, W1.x, W1.y, W1.z, W2.x, W2.y, W2.z};
#pragma unroll
    for (int i = 0; i < kFaceTerms; ++i) T[i] = values[i];
}

// 2^-e for the binary exponent e of `largest` (> 0), built from its exponent field: scaling by
// it is exact, so a far-field gradient is brought to O(1) without a division's rounding before
// its squared length is formed (kernels/predicates.py:719 stable_normalize divides by the
// largest component instead). Exponent fields are clamped to [1, 2045] so the scale is a normal
// number; a subnormal `largest` is then scaled by 2^1022, which keeps its square representable.
__device__ __forceinline__ double inverse_power_of_two(double largest) {
    long long e = (__double_as_longlong(largest) >> 52) & 0x7ff;
    e = e < 1 ? 1 : (e > 2045 ? 2045 : e);
    return __longlong_as_double((2046 - e) << 52);
}

// -div of the unit gradient at (vertex, column) from the per-face terms, summed over the vertex's
// corners in ascending slot order: d_e = (W_e . s) / |s| with s = g 2^-e the rescaled gradient.
// A thread takes CP adjacent columns of one vertex, so the per-corner index and term loads are
// shared by CP columns (with CP > 1 the strides are even and u, out 16-byte aligned: u is read
// and out written as double2). Columns from n_columns up are written as zero.
// CP = 4 is held to 64 registers a thread (4 blocks of 256 an SM instead of 3; a few bytes
// spill to L1): 3.15 -> 2.91 ms on a 2.6M-vertex mesh at 64 columns.
template <int CP>
__global__ void __launch_bounds__(256, CP == 4 ? 4 : 1) grad_div_terms_kernel(const double* __restrict__ terms, const int* __restrict__ faces,
                                      const int* __restrict__ corner_offsets,
                                      const int* __restrict__ corner_slots, int n, int k,
                                      const double* __restrict__ u, int u_stride,
                                      const int* __restrict__ u_iperm, double* __restrict__ out,
                                      int out_stride, const int* __restrict__ out_iperm,
                                      const char* __restrict__ out_pinned) {
    const int groups = out_stride / CP;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * groups) return;
    const int v = (int)(t / groups), c0 = (int)(t % groups) * CP;
    const int row = row_of(out_iperm, v);
    double acc[CP];
#pragma unroll
    for (int j = 0; j < CP; ++j) acc[j] = 0.0;
    auto load = [&](int r, double* dst) {
        const double* src = u + (size_t)r * u_stride + c0;
        if (CP == 1) {
            dst[0] = src[0];
        } else {
#pragma unroll
            for (int j = 0; j < CP; j += 2) {
                // A pair starting below k lies inside the row (even strides).
                const double2 p = (c0 + j < k) ? *reinterpret_cast<const double2*>(src + j) : make_double2(0.0, 0.0);
                dst[j] = p.x;
                dst[j + 1] = p.y;
            }
        }
    };
    if (c0 < k) {
        const int end = corner_offsets[v + 1];
        for (int p = corner_offsets[v]; p < end; ++p) {
            const int q = corner_slots[p];
            const int f = q / 3, e = q - 3 * f;
            double u0[CP], u1[CP], u2[CP];
            load(row_of(u_iperm, faces[3 * f]), u0);
            load(row_of(u_iperm, faces[3 * f + 1]), u1);
            load(row_of(u_iperm, faces[3 * f + 2]), u2);
            const double* T = terms + (size_t)kFaceTerms * f;
            const double a0 = T[0], a1 = T[1], a2 = T[2], b0 = T[3], b1 = T[4], b2 = T[5];
            const double w0 = T[6], w1 = T[7], w2 = T[8];
            const double* W = T + 9 + 3 * e;
            const double W0 = W[0], W1 = W[1], W2 = W[2];
#pragma unroll
            for (int j = 0; j < CP; ++j) {
                const double gx = fma(u0[j], a0, fma(u1[j], b0, u2[j] * w0));
                const double gy = fma(u0[j], a1, fma(u1[j], b1, u2[j] * w1));
                const double gz = fma(u0[j], a2, fma(u1[j], b2, u2[j] * w2));
                const double largest = fmax(fabs(gx), fmax(fabs(gy), fabs(gz)));
                if (largest == 0.0) continue;  // no gradient: the unit gradient is zero
                const double scale = inverse_power_of_two(largest);
                const double sx = gx * scale, sy = gy * scale, sz = gz * scale;
                const double along = fma(sx, W0, fma(sy, W1, sz * W2));
                acc[j] += along * rsqrt(fma(sx, sx, fma(sy, sy, sz * sz)));
            }
        }
    }
    const bool pinned = out_pinned && out_pinned[row];
    double* o = out + (size_t)row * out_stride + c0;
#pragma unroll
    for (int j = 0; j < CP; ++j)
        if (pinned || c0 + j >= k) acc[j] = 0.0;
    if (CP == 1) {
        o[0] = acc[0];
    } else {
#pragma unroll
        for (int j = 0; j < CP; j += 2) *reinterpret_cast<double2*>(o + j) = make_double2(acc[j], acc[j + 1]);
    }
}

// ---- The divergence over corner records ----------------------------------------------------
// The per-corner form above reads, at each corner, its slot, its face's three vertices and twelve
// of the face's eighteen terms through that slot: 16 loads a corner, each behind the slot's. The
// records copy, once per face buffer and corner index, each corner's twelve terms (the face's
// gradient bases a, b, w and the corner's W_e) into 96 contiguous bytes and its face's vertices
// into an int4, both in the corner index's order: a vertex's corners are then consecutive records,
// read as six 16-byte loads and one (no slot indirection). The arithmetic and the corner order are
// the per-corner form's, so the results are its bits.
constexpr int kRecordPairs = 6;  // double2 a record: a0 a1 | a2 b0 | b1 b2 | w0 w1 | w2 W0 | W1 W2

__global__ void corner_records_kernel(const double* __restrict__ terms, const int* __restrict__ faces,
                                      const int* __restrict__ corner_slots, long long n_corners,
                                      double2* __restrict__ records, int4* __restrict__ ids) {
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= n_corners) return;
    const int q = corner_slots[p];
    const int f = q / 3, e = q - 3 * f;
    const double* T = terms + (size_t)kFaceTerms * f;
    const double* W = T + 9 + 3 * e;
    double2* R = records + (size_t)kRecordPairs * p;
    R[0] = make_double2(T[0], T[1]);
    R[1] = make_double2(T[2], T[3]);
    R[2] = make_double2(T[4], T[5]);
    R[3] = make_double2(T[6], T[7]);
    R[4] = make_double2(T[8], W[0]);
    R[5] = make_double2(W[1], W[2]);
    ids[p] = make_int4(faces[3 * f], faces[3 * f + 1], faces[3 * f + 2], 0);
}

template <int CP>
__global__ void __launch_bounds__(256, CP == 4 ? 4 : 1)
grad_div_records_kernel(const double2* __restrict__ records, const int4* __restrict__ ids,
                        const int* __restrict__ corner_offsets, int n, int k, const double* __restrict__ u,
                        int u_stride, const int* __restrict__ u_iperm, double* __restrict__ out, int out_stride,
                        const int* __restrict__ out_iperm, const char* __restrict__ out_pinned) {
    const int groups = out_stride / CP;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n * groups) return;
    const int v = (int)(t / groups), c0 = (int)(t % groups) * CP;
    const int row = row_of(out_iperm, v);
    double acc[CP];
#pragma unroll
    for (int j = 0; j < CP; ++j) acc[j] = 0.0;
    auto load = [&](int r, double* dst) {
        const double* src = u + (size_t)r * u_stride + c0;
        if (CP == 1) {
            dst[0] = src[0];
        } else {
#pragma unroll
            for (int j = 0; j < CP; j += 2) {
                // A pair starting below k lies inside the row (even strides).
                const double2 p = (c0 + j < k) ? *reinterpret_cast<const double2*>(src + j) : make_double2(0.0, 0.0);
                dst[j] = p.x;
                dst[j + 1] = p.y;
            }
        }
    };
    if (c0 < k) {
        const int end = corner_offsets[v + 1];
        for (int p = corner_offsets[v]; p < end; ++p) {
            const int4 id = ids[p];
            double u0[CP], u1[CP], u2[CP];
            load(row_of(u_iperm, id.x), u0);
            load(row_of(u_iperm, id.y), u1);
            load(row_of(u_iperm, id.z), u2);
            const double2* R = records + (size_t)kRecordPairs * p;
            const double2 r0 = R[0], r1 = R[1], r2 = R[2], r3 = R[3], r4 = R[4], r5 = R[5];
            const double a0 = r0.x, a1 = r0.y, a2 = r1.x, b0 = r1.y, b1 = r2.x, b2 = r2.y;
            const double w0 = r3.x, w1 = r3.y, w2 = r4.x, W0 = r4.y, W1 = r5.x, W2 = r5.y;
#pragma unroll
            for (int j = 0; j < CP; ++j) {
                const double gx = fma(u0[j], a0, fma(u1[j], b0, u2[j] * w0));
                const double gy = fma(u0[j], a1, fma(u1[j], b1, u2[j] * w1));
                const double gz = fma(u0[j], a2, fma(u1[j], b2, u2[j] * w2));
                const double largest = fmax(fabs(gx), fmax(fabs(gy), fabs(gz)));
                if (largest == 0.0) continue;  // no gradient: the unit gradient is zero
                const double scale = inverse_power_of_two(largest);
                const double sx = gx * scale, sy = gy * scale, sz = gz * scale;
                const double along = fma(sx, W0, fma(sy, W1, sz * W2));
                acc[j] += along * rsqrt(fma(sx, sx, fma(sy, sy, sz * sz)));
            }
        }
    }
    const bool pinned = out_pinned && out_pinned[row];
    double* o = out + (size_t)row * out_stride + c0;
#pragma unroll
    for (int j = 0; j < CP; ++j)
        if (pinned || c0 + j >= k) acc[j] = 0.0;
    if (CP == 1) {
        o[0] = acc[0];
    } else {
#pragma unroll
        for (int j = 0; j < CP; j += 2) *reinterpret_cast<double2*>(o + j) = make_double2(acc[j], acc[j + 1]);
    }
}

// ---- The divergence face by face over tiles of vertices ------------------------------------
// The per-corner form above recomputes a face's unit gradient at each of its three corners. Here
// a CTA takes kTileVertices consecutive vertices, forms the unit gradient of each distinct face
// they touch once per column (into shared memory, as its three corner contributions d_e), then
// sums each vertex's corners from there in ascending slot order: the same terms in the same
// order, a third of the gradients, normalisations and reciprocal square roots.
constexpr int kTileVertices = 32;   // vertices a tile
constexpr int kTileColumns = 16;    // columns a pass over a tile's faces takes
constexpr int kTileFaces = 192;     // distinct faces a tile holds in shared memory
constexpr int kTileCorners = 1024;  // corners the set-up deduplicates in shared memory
constexpr int kTileSmem = kTileFaces * 3 * kTileColumns * (int)sizeof(double);

// Set-up, once per face buffer and corner index: tile t's distinct faces in first-corner order,
// stored over the start of the tile's own corner range of tile_faces (a tile has no more distinct
// faces than corners), their count (-1 past kTileCorners corners or kTileFaces faces: the
// divergence takes the per-corner form on such a tile), and each corner's code, its face's place
// in the list times 3 plus its corner.
__global__ void __launch_bounds__(256) divergence_tiles_kernel(const int* __restrict__ corner_offsets,
                                                               const int* __restrict__ corner_slots, int n,
                                                               int* __restrict__ tile_faces,
                                                               int* __restrict__ tile_counts,
                                                               int* __restrict__ corner_codes) {
    __shared__ int face[kTileCorners];
    __shared__ int first[kTileCorners];
    const int t = blockIdx.x;
    const int v0 = t * kTileVertices, v1 = min(n, v0 + kTileVertices);
    const int p0 = corner_offsets[v0], m = corner_offsets[v1] - p0;
    if (m > kTileCorners) {
        if (threadIdx.x == 0) tile_counts[t] = -1;
        return;
    }
    for (int i = threadIdx.x; i < m; i += blockDim.x) face[i] = corner_slots[p0 + i] / 3;
    __syncthreads();
    // Each corner's first corner of the same face in the tile.
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int f = face[i];
        int j = 0;
        while (face[j] != f) ++j;
        first[i] = j;
    }
    __syncthreads();
    // Places in first-corner order (one thread: a few hundred corners, once per mesh); a first
    // corner's entry becomes -(place + 1).
    if (threadIdx.x == 0) {
        int count = 0;
        for (int i = 0; i < m; ++i)
            if (first[i] == i) {
                tile_faces[p0 + count] = face[i];
                first[i] = -(count + 1);
                ++count;
            }
        tile_counts[t] = count > kTileFaces ? -1 : count;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int j = first[i];
        const int place = j < 0 ? -j - 1 : -first[j] - 1;
        corner_codes[p0 + i] = 3 * place + corner_slots[p0 + i] % 3;
    }
}

// The unit gradient of face f at column c, as its three corner contributions d_e = (W_e . s) / |s|
// (zero where the gradient is zero): the arithmetic of grad_div_terms_kernel.
__device__ __forceinline__ void face_contributions(const double* __restrict__ T, double u0, double u1, double u2,
                                                   double* d) {
    const double gx = fma(u0, T[0], fma(u1, T[3], u2 * T[6]));
    const double gy = fma(u0, T[1], fma(u1, T[4], u2 * T[7]));
    const double gz = fma(u0, T[2], fma(u1, T[5], u2 * T[8]));
    const double largest = fmax(fabs(gx), fmax(fabs(gy), fabs(gz)));
    if (largest == 0.0) {
        d[0] = d[1] = d[2] = 0.0;
        return;
    }
    const double scale = inverse_power_of_two(largest);
    const double sx = gx * scale, sy = gy * scale, sz = gz * scale;
    const double r = rsqrt(fma(sx, sx, fma(sy, sy, sz * sz)));
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const double* W = T + 9 + 3 * e;
        d[e] = fma(sx, W[0], fma(sy, W[1], sz * W[2])) * r;
    }
}

__global__ void __launch_bounds__(256) grad_div_tiled_kernel(
    const double* __restrict__ terms, const int* __restrict__ faces, const int* __restrict__ corner_offsets,
    const int* __restrict__ corner_slots, const int* __restrict__ tile_faces, const int* __restrict__ tile_counts,
    const int* __restrict__ corner_codes, int n, int k, const double* __restrict__ u, int u_stride,
    const int* __restrict__ u_iperm, double* __restrict__ out, int out_stride, const int* __restrict__ out_iperm,
    const char* __restrict__ out_pinned) {
    extern __shared__ double contributions[];  // [place * 3 + corner][column of the pass]
    const int t = blockIdx.x;
    const int v0 = t * kTileVertices, v1 = min(n, v0 + kTileVertices);
    const int count = tile_counts[t];
    if (count < 0) {
        // A crowded tile: each (vertex, column) sums its corners' own gradients.
        for (int item = threadIdx.x; item < (v1 - v0) * out_stride; item += blockDim.x) {
            const int v = v0 + item / out_stride, c = item % out_stride;
            double acc = 0.0;
            if (c < k)
                for (int p = corner_offsets[v]; p < corner_offsets[v + 1]; ++p) {
                    const int q = corner_slots[p], f = q / 3, e = q - 3 * f;
                    double d[3];
                    face_contributions(terms + (size_t)kFaceTerms * f,
                                       u[(size_t)row_of(u_iperm, faces[3 * f]) * u_stride + c],
                                       u[(size_t)row_of(u_iperm, faces[3 * f + 1]) * u_stride + c],
                                       u[(size_t)row_of(u_iperm, faces[3 * f + 2]) * u_stride + c], d);
                    acc += d[e];
                }
            const int row = row_of(out_iperm, v);
            out[(size_t)row * out_stride + c] = ((out_pinned && out_pinned[row]) || c >= k) ? 0.0 : acc;
        }
        return;
    }
    const int p0 = corner_offsets[v0];
    for (int c0 = 0; c0 < out_stride; c0 += kTileColumns) {
        for (int item = threadIdx.x; item < count * kTileColumns; item += blockDim.x) {
            const int place = item / kTileColumns, j = item % kTileColumns, c = c0 + j;
            double d[3] = {0.0, 0.0, 0.0};
            if (c < k) {
                const int f = tile_faces[p0 + place];
                face_contributions(terms + (size_t)kFaceTerms * f,
                                   u[(size_t)row_of(u_iperm, faces[3 * f]) * u_stride + c],
                                   u[(size_t)row_of(u_iperm, faces[3 * f + 1]) * u_stride + c],
                                   u[(size_t)row_of(u_iperm, faces[3 * f + 2]) * u_stride + c], d);
            }
#pragma unroll
            for (int e = 0; e < 3; ++e) contributions[(3 * place + e) * kTileColumns + j] = d[e];
        }
        __syncthreads();
        const int width = min(kTileColumns, out_stride - c0);
        for (int item = threadIdx.x; item < (v1 - v0) * kTileColumns; item += blockDim.x) {
            const int v = v0 + item / kTileColumns, j = item % kTileColumns, c = c0 + j;
            if (j >= width) continue;
            double acc = 0.0;
            const int end = corner_offsets[v + 1];
            for (int p = corner_offsets[v]; p < end; ++p) acc += contributions[corner_codes[p] * kTileColumns + j];
            const int row = row_of(out_iperm, v);
            out[(size_t)row * out_stride + c] = ((out_pinned && out_pinned[row]) || c >= k) ? 0.0 : acc;
        }
        __syncthreads();
    }
}

int allow_tile_memory() {
    static int allowed[64] = {};
    int device = 0;
    OB_CUDA(cudaGetDevice(&device));
    if (device >= 0 && device < 64 && allowed[device]) return OB_OK;
    OB_CUDA(cudaFuncSetAttribute(grad_div_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
    if (device >= 0 && device < 64) allowed[device] = 1;
    return OB_OK;
}

// Seeds of k source sets in a factor's numbering: rhs (stride `stride`, zeroed first) gets 1 at
// each source's row, 0 at pinned rows.
__global__ void seed_permuted_kernel(const int* __restrict__ sources,
                                     const int* __restrict__ source_offsets, int k,
                                     const int* __restrict__ iperm, const char* __restrict__ pinned,
                                     int stride, double* __restrict__ rhs) {
    const int c = blockIdx.y;
    for (int i = source_offsets[c] + threadIdx.x; i < source_offsets[c + 1]; i += blockDim.x) {
        const int row = iperm[sources[i]];
        if (!pinned[row]) rhs[(size_t)row * stride + c] = 1.0;
    }
}

// Per column: the sum of phi over every row and over the column's sources. The whole-field sums
// read rows whole (a row's columns are contiguous): thread t of a block owns column t % stride
// (blockDim a multiple of stride), a block's per-column partials are added in thread order, then
// across blocks in block order by the last block to finish. The source sums are a handful of
// rows, added by that last block.
__global__ void shift_sums_kernel(const double* __restrict__ phi, int n, int stride,
                                  const int* __restrict__ iperm, const int* __restrict__ sources,
                                  const int* __restrict__ source_offsets, int k, int orient,
                                  double* __restrict__ partials, unsigned int* counter,
                                  double2* __restrict__ sums) {
    __shared__ double tree[kThreads];
    __shared__ int last;
    const int c = threadIdx.x % stride;
    double everywhere = 0.0;
    const long long total = (long long)n * stride;
    const long long step = (long long)gridDim.x * blockDim.x;  // a multiple of stride
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    // Eight independent loads in flight a thread (the sum stays in index order per thread).
    for (; t + 7 * step < total; t += 8 * step) {
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = phi[t + q * step];
#pragma unroll
        for (int q = 0; q < 8; ++q) everywhere += v[q];
    }
    for (; t < total; t += step) everywhere += phi[t];
    tree[threadIdx.x] = everywhere;
    __syncthreads();
    if ((int)threadIdx.x < stride) {
        double column = 0.0;
        for (int t = threadIdx.x; t < (int)blockDim.x; t += stride) column += tree[t];
        partials[(size_t)blockIdx.x * stride + threadIdx.x] = column;
    }
    if (!last_block_arrived(counter, &last)) return;
    // The last block: thread t folds column t % stride over blocks t / stride, t / stride + groups,
    // ... in order; the groups' sums then meet in group order (a fixed order for a launch shape).
    const int groups = blockDim.x / stride;
    // Four running sums (blocks b, b + groups, b + 2 groups, b + 3 groups of each round) so four
    // loads are in flight, added together in a fixed order at the end.
    double part4[4] = {0.0, 0.0, 0.0, 0.0};
    int bx = threadIdx.x / stride;
    for (; bx + 3 * groups < (int)gridDim.x; bx += 4 * groups)
#pragma unroll
        for (int q = 0; q < 4; ++q) part4[q] += __ldcg(&partials[(size_t)(bx + q * groups) * stride + c]);
    for (int q = 0; bx < (int)gridDim.x; bx += groups, ++q) part4[q] += __ldcg(&partials[(size_t)bx * stride + c]);
    const double part = (part4[0] + part4[1]) + (part4[2] + part4[3]);
    __syncthreads();
    tree[threadIdx.x] = part;
    __syncthreads();
    for (int col = threadIdx.x; col < k; col += blockDim.x) {
        double g = 0.0;
        for (int q = 0; q < groups; ++q) g += tree[q * stride + col];
        double s = 0.0;
        for (int i = source_offsets[col]; i < source_offsets[col + 1]; ++i)
            s += __ldcg(&phi[(size_t)iperm[sources[i]] * stride + col]);
        // The column's shift (the mean over its sources) and orientation: flipped (-1) when the
        // whole field's mean lies below the shift.
        const double offset = s / (double)(source_offsets[col + 1] - source_offsets[col]);
        const double flip = (orient != 0 && g / (double)n - offset < 0.0) ? -1.0 : 1.0;
        sums[col] = make_double2(offset, flip);
    }
}

// out[c][v] = the shifted, oriented phi of vertex v in column c (ordito/kernels/heat.py:3406).
__global__ void shift_out_kernel(const double* __restrict__ phi, int n, int stride,
                                 const int* __restrict__ iperm, const double2* __restrict__ shifts,
                                 int k, double* __restrict__ out) {
    __shared__ double tile[32][33];
    // Tile of 32 vertices x 32 columns: read along columns (a factor row), write along vertices.
    const int v0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int v = v0 + i, c = c0 + threadIdx.x;
        if (v < n && c < k) tile[i][threadIdx.x] = phi[(size_t)iperm[v] * stride + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, v = v0 + threadIdx.x;
        if (v >= n || c >= k) continue;
        const double2 s = shifts[c];  // (offset, +1 or -1): offset - value exactly when flipped
        out[(size_t)c * n + v] = s.y * (tile[threadIdx.x][i] - s.x);
    }
}

// Packed meshes (many meshes as one block-diagonal system, column c = every mesh's c-th
// single-source query): per (mesh, column) the sum of phi over the mesh's rows and phi at the
// query's source. Each mesh's rows are cut into chunks of kPackedChunk (a block a chunk, so a
// large mesh is summed by many blocks and the grid does not wait on the largest mesh), each
// chunk's per-column sums written apart, then folded per mesh in chunk order: a fixed order for a
// given packing.
constexpr int kPackedChunk = 2048;

// The chunk table: chunk_first[m] = mesh m's first chunk (chunk_first[n_meshes] = the count) and
// per chunk (mesh, first row, end row). One block; the meshes' chunk counts are scanned in
// order, kThreads meshes at a time.
__global__ void packed_chunks_kernel(const int* __restrict__ vertex_offsets, int n_meshes,
                                     int* __restrict__ chunk_first, int4* __restrict__ chunks) {
    __shared__ int scan[kThreads];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n_meshes; base += blockDim.x) {
        const int m = base + threadIdx.x;
        const int v0 = m < n_meshes ? vertex_offsets[m] : 0, v1 = m < n_meshes ? vertex_offsets[m + 1] : 0;
        const int count = (v1 - v0 + kPackedChunk - 1) / kPackedChunk;
        scan[threadIdx.x] = count;
        __syncthreads();
        for (int d = 1; d < (int)blockDim.x; d <<= 1) {  // inclusive scan (Hillis-Steele)
            const int add = threadIdx.x >= (unsigned)d ? scan[threadIdx.x - d] : 0;
            __syncthreads();
            scan[threadIdx.x] += add;
            __syncthreads();
        }
        const int first = carry + scan[threadIdx.x] - count;
        if (m < n_meshes) {
            chunk_first[m] = first;
            for (int j = 0; j < count; ++j)
                chunks[first + j] = make_int4(m, v0 + j * kPackedChunk, min(v1, v0 + (j + 1) * kPackedChunk), 0);
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += scan[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) chunk_first[n_meshes] = carry;
}

// A chunk's per-column sums of phi: threads own column t % stride (blockDim a multiple of
// stride), rows t / stride + j (blockDim / stride) in order, then the row groups added in order.
__global__ void packed_partials_kernel(const double* __restrict__ phi, int stride, const int* __restrict__ iperm,
                                       const int* __restrict__ chunk_first, int n_meshes,
                                       const int4* __restrict__ chunks, double* __restrict__ partials) {
    __shared__ double tree[kThreads];
    if ((int)blockIdx.x >= chunk_first[n_meshes]) return;
    const int4 chunk = chunks[blockIdx.x];
    const int c = threadIdx.x % stride, rows_per_pass = blockDim.x / stride;
    double total = 0.0;
    for (int v = chunk.y + threadIdx.x / stride; v < chunk.z; v += rows_per_pass)
        total += phi[(size_t)row_of(iperm, v) * stride + c];
    tree[threadIdx.x] = total;
    __syncthreads();
    if ((int)threadIdx.x < stride) {
        double column = 0.0;
        for (int t = threadIdx.x; t < (int)blockDim.x; t += stride) column += tree[t];
        partials[(size_t)blockIdx.x * stride + threadIdx.x] = column;
    }
}

// sums[m][c] = (phi at mesh m's c-th source, or 0 without one; the mesh's chunks' sums in chunk
// order): a block a mesh, a thread a column.
__global__ void packed_fold_kernel(const double* __restrict__ phi, int stride, const int* __restrict__ iperm,
                                   const int* __restrict__ vertex_offsets, const int* __restrict__ sources, int k,
                                   const int* __restrict__ chunk_first, const double* __restrict__ partials,
                                   double2* __restrict__ sums) {
    const int m = blockIdx.x;
    for (int c = threadIdx.x; c < k; c += blockDim.x) {
        double column = 0.0;
        for (int b = chunk_first[m]; b < chunk_first[m + 1]; ++b) column += partials[(size_t)b * stride + c];
        const int s = sources[(size_t)m * k + c];
        const double at = s >= 0 ? phi[(size_t)row_of(iperm, vertex_offsets[m] + s) * stride + c] : 0.0;
        sums[(size_t)m * k + c] = make_double2(at, column);
    }
}

// out[c][v]: the shifted, oriented phi of vertex v in column c (kernels/heat.py:3406 per mesh);
// zero where v's mesh has no query in column c. Tiles of 32 vertices x 32 columns: phi read along
// a row's columns, out written along vertices, each vertex's mesh found once a tile.
__global__ void shift_packed_out_kernel(const double* __restrict__ phi, int n, int stride,
                                        const int* __restrict__ iperm, const int* __restrict__ vertex_offsets,
                                        int n_meshes, const int* __restrict__ sources, int k,
                                        const double2* __restrict__ sums, double* __restrict__ out) {
    __shared__ double tile[32][33];
    __shared__ int mesh_of[32];
    const int v0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    if (threadIdx.y == 0) {
        const int v = v0 + threadIdx.x;
        int lo = 0, hi = n_meshes - 1;  // the mesh holding v: vertex_offsets[m] <= v < [m + 1]
        if (v < n)
            while (lo < hi) {
                const int mid = (lo + hi + 1) / 2;
                if (vertex_offsets[mid] <= v) lo = mid;
                else hi = mid - 1;
            }
        mesh_of[threadIdx.x] = lo;
    }
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int v = v0 + i, c = c0 + threadIdx.x;
        if (v < n && c < k) tile[i][threadIdx.x] = phi[(size_t)row_of(iperm, v) * stride + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, v = v0 + threadIdx.x;
        if (v >= n || c >= k) continue;
        const int m = mesh_of[threadIdx.x];
        double shifted = 0.0;
        if (sources[(size_t)m * k + c] >= 0) {
            const double2 s = sums[(size_t)m * k + c];
            const double value = tile[threadIdx.x][i];
            const int count = vertex_offsets[m + 1] - vertex_offsets[m];
            shifted = (s.y / (double)count - s.x < 0.0) ? s.x - value : value - s.x;
        }
        out[(size_t)c * n + v] = shifted;
    }
}

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_corner_index_workspace(int n_vertices, int n_faces, size_t* bytes) {
    OB_REQUIRE(bytes && n_vertices >= 0 && n_faces >= 0, "ob_corner_index_workspace: bad argument");
    const int corners = 3 * n_faces;
    size_t sort_bytes = 0;
    if (corners > 0)
        OB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const int*)nullptr, (int*)nullptr,
                                                (const int*)nullptr, (int*)nullptr, corners));
    *bytes = align_up(sort_bytes) + 3 * align_up(sizeof(int) * (size_t)std::max(corners, 1)) + 256;
    return OB_OK;
}

int ob_renumber(const int32_t* indices, long long count, const int32_t* map, int32_t* out,
                ob_stream_t stream) {
    OB_REQUIRE(count >= 0, "ob_renumber: negative count");
    if (count == 0) return OB_OK;
    OB_REQUIRE(indices && map && out, "ob_renumber: null pointer");
    const int blocks = (int)std::min<long long>((count + kThreads - 1) / kThreads, 8LL * sm_count());
    renumber_kernel<<<blocks, kThreads, 0, as_stream(stream)>>>(indices, count, map, out);
    OB_CHECK_LAUNCH("renumber");
    return OB_OK;
}

int ob_corner_index(const int32_t* faces, int n_faces, int n_vertices, int32_t* corner_offsets,
                    int32_t* corner_slots, void* workspace, size_t workspace_bytes,
                    ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(corner_offsets && n_vertices >= 0 && n_faces >= 0, "ob_corner_index: bad argument");
    const int corners = 3 * n_faces;
    if (corners == 0) {
        OB_CUDA(cudaMemsetAsync(corner_offsets, 0, sizeof(int) * (size_t)(n_vertices + 1), stream));
        return OB_OK;
    }
    OB_REQUIRE(faces && corner_slots && workspace, "ob_corner_index: null pointer");
    size_t needed = 0;
    int st = ob_corner_index_workspace(n_vertices, n_faces, &needed);
    if (st) return st;
    OB_REQUIRE(workspace_bytes >= needed, "ob_corner_index: workspace of %zu bytes, %zu needed",
               workspace_bytes, needed);
    char* ws = reinterpret_cast<char*>(align_up(reinterpret_cast<size_t>(workspace)));
    const size_t vec = align_up(sizeof(int) * (size_t)corners);
    int* keys_in = reinterpret_cast<int*>(ws);
    int* slots_in = reinterpret_cast<int*>(ws + vec);
    int* keys_out = reinterpret_cast<int*>(ws + 2 * vec);
    void* sort_temp = ws + 3 * vec;
    size_t sort_bytes = workspace_bytes - 256 - 3 * vec;
    corner_keys_kernel<<<ceil_div(corners, kThreads), kThreads, 0, stream>>>(faces, corners,
                                                                             n_vertices, keys_in,
                                                                             slots_in);
    OB_CHECK_LAUNCH("corner_keys");
    int bits = 1;
    while ((1LL << bits) <= (long long)n_vertices) ++bits;
    OB_CUDA(cub::DeviceRadixSort::SortPairs(sort_temp, sort_bytes, keys_in, keys_out, slots_in,
                                            corner_slots, corners, 0, bits, stream));
    count_launch();
    corner_offsets_kernel<<<ceil_div(corners + 1, kThreads), kThreads, 0, stream>>>(
        keys_out, corners, n_vertices, corner_offsets);
    OB_CHECK_LAUNCH("corner_offsets");
    return OB_OK;
}

int ob_grad_div_gather(const float* xyz, const int32_t* faces, const float* normals,
                       const float* areas, const float* cot, const int32_t* corner_offsets,
                       const int32_t* corner_slots, int n_vertices, int n_columns, const double* u,
                       int u_stride, const int32_t* u_iperm, double* out, int out_stride,
                       const int32_t* out_iperm, const char* out_pinned, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && n_columns >= 1 && u_stride >= n_columns && out_stride >= n_columns,
               "ob_grad_div_gather: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(xyz && faces && normals && areas && cot && corner_offsets && corner_slots && u && out,
               "ob_grad_div_gather: null pointer");
    const long long total = (long long)n_vertices * out_stride;
    grad_div_gather_kernel<<<ceil_div(total, kThreads), kThreads, 0, stream>>>(
        xyz, faces, normals, areas, cot, corner_offsets, corner_slots, n_vertices, n_columns, u,
        u_stride, u_iperm, out, out_stride, out_iperm, out_pinned);
    OB_CHECK_LAUNCH("grad_div_gather");
    return OB_OK;
}

int ob_face_gradient_terms(const float* xyz, const int32_t* faces, int n_faces, const float* normals,
                           const float* areas, const float* cot, double* terms, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 0, "ob_face_gradient_terms: bad size");
    if (n_faces == 0) return OB_OK;
    OB_REQUIRE(xyz && faces && normals && areas && cot && terms, "ob_face_gradient_terms: null pointer");
    face_gradient_terms_kernel<<<ceil_div(n_faces, kThreads), kThreads, 0, stream>>>(
        xyz, faces, n_faces, normals, areas, cot, terms);
    OB_CHECK_LAUNCH("face_gradient_terms");
    return OB_OK;
}

int ob_grad_div_terms(const double* terms, const int32_t* faces, const int32_t* corner_offsets,
                      const int32_t* corner_slots, int n_vertices, int n_columns, const double* u,
                      int u_stride, const int32_t* u_iperm, double* out, int out_stride,
                      const int32_t* out_iperm, const char* out_pinned, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && n_columns >= 1 && u_stride >= n_columns && out_stride >= n_columns,
               "ob_grad_div_terms: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(terms && faces && corner_offsets && corner_slots && u && out, "ob_grad_div_terms: null pointer");
    // Columns a thread takes: 4 or 2 when the strides and pointers allow paired loads and stores.
    const bool paired = u_stride % 2 == 0 && out_stride % 2 == 0 && ((uintptr_t)u & 15) == 0 &&
                        ((uintptr_t)out & 15) == 0;
    const int cp = !paired ? 1 : (out_stride % 4 == 0 ? 4 : 2);
    const long long total = (long long)n_vertices * (out_stride / cp);
    const int blocks = (int)ceil_div(total, kThreads);
    if (cp == 4)
        grad_div_terms_kernel<4><<<blocks, kThreads, 0, stream>>>(terms, faces, corner_offsets, corner_slots,
                                                                  n_vertices, n_columns, u, u_stride, u_iperm,
                                                                  out, out_stride, out_iperm, out_pinned);
    else if (cp == 2)
        grad_div_terms_kernel<2><<<blocks, kThreads, 0, stream>>>(terms, faces, corner_offsets, corner_slots,
                                                                  n_vertices, n_columns, u, u_stride, u_iperm,
                                                                  out, out_stride, out_iperm, out_pinned);
    else
        grad_div_terms_kernel<1><<<blocks, kThreads, 0, stream>>>(terms, faces, corner_offsets, corner_slots,
                                                                  n_vertices, n_columns, u, u_stride, u_iperm,
                                                                  out, out_stride, out_iperm, out_pinned);
    OB_CHECK_LAUNCH("grad_div_terms");
    return OB_OK;
}

int ob_corner_records(const double* terms, const int32_t* faces, const int32_t* corner_slots, int n_faces,
                      double* records, int32_t* ids, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 0, "ob_corner_records: bad size");
    if (n_faces == 0) return OB_OK;
    OB_REQUIRE(terms && faces && corner_slots && records && ids, "ob_corner_records: null pointer");
    OB_REQUIRE(((uintptr_t)records & 15) == 0 && ((uintptr_t)ids & 15) == 0,
               "ob_corner_records: records and ids must start on 16 bytes");
    const long long corners = 3LL * n_faces;
    corner_records_kernel<<<ceil_div(corners, kThreads), kThreads, 0, stream>>>(
        terms, faces, corner_slots, corners, reinterpret_cast<double2*>(records), reinterpret_cast<int4*>(ids));
    OB_CHECK_LAUNCH("corner_records");
    return OB_OK;
}

int ob_grad_div_records(const double* records, const int32_t* ids, const int32_t* corner_offsets, int n_vertices,
                        int n_columns, const double* u, int u_stride, const int32_t* u_iperm, double* out,
                        int out_stride, const int32_t* out_iperm, const char* out_pinned, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && n_columns >= 1 && u_stride >= n_columns && out_stride >= n_columns,
               "ob_grad_div_records: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(records && ids && corner_offsets && u && out, "ob_grad_div_records: null pointer");
    OB_REQUIRE(((uintptr_t)records & 15) == 0 && ((uintptr_t)ids & 15) == 0,
               "ob_grad_div_records: records and ids must start on 16 bytes");
    const bool paired = u_stride % 2 == 0 && out_stride % 2 == 0 && ((uintptr_t)u & 15) == 0 &&
                        ((uintptr_t)out & 15) == 0;
    const int cp = !paired ? 1 : (out_stride % 4 == 0 ? 4 : 2);
    const long long total = (long long)n_vertices * (out_stride / cp);
    const int blocks = (int)ceil_div(total, kThreads);
    const double2* R = reinterpret_cast<const double2*>(records);
    const int4* I = reinterpret_cast<const int4*>(ids);
    if (cp == 4)
        grad_div_records_kernel<4><<<blocks, kThreads, 0, stream>>>(R, I, corner_offsets, n_vertices, n_columns, u,
                                                                    u_stride, u_iperm, out, out_stride, out_iperm,
                                                                    out_pinned);
    else if (cp == 2)
        grad_div_records_kernel<2><<<blocks, kThreads, 0, stream>>>(R, I, corner_offsets, n_vertices, n_columns, u,
                                                                    u_stride, u_iperm, out, out_stride, out_iperm,
                                                                    out_pinned);
    else
        grad_div_records_kernel<1><<<blocks, kThreads, 0, stream>>>(R, I, corner_offsets, n_vertices, n_columns, u,
                                                                    u_stride, u_iperm, out, out_stride, out_iperm,
                                                                    out_pinned);
    OB_CHECK_LAUNCH("grad_div_records");
    return OB_OK;
}

int ob_divergence_tiles(const int32_t* corner_offsets, const int32_t* corner_slots, int n_vertices,
                        int32_t* tile_faces, int32_t* tile_counts, int32_t* corner_codes, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0, "ob_divergence_tiles: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(corner_offsets && corner_slots && tile_faces && tile_counts && corner_codes,
               "ob_divergence_tiles: null pointer");
    divergence_tiles_kernel<<<ceil_div(n_vertices, kTileVertices), 256, 0, stream>>>(
        corner_offsets, corner_slots, n_vertices, tile_faces, tile_counts, corner_codes);
    OB_CHECK_LAUNCH("divergence tiles");
    return OB_OK;
}

int ob_grad_div_tiled(const double* terms, const int32_t* faces, const int32_t* corner_offsets,
                      const int32_t* corner_slots, const int32_t* tile_faces, const int32_t* tile_counts,
                      const int32_t* corner_codes, int n_vertices, int n_columns, const double* u, int u_stride,
                      const int32_t* u_iperm, double* out, int out_stride, const int32_t* out_iperm,
                      const char* out_pinned, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && n_columns >= 1 && u_stride >= n_columns && out_stride >= n_columns,
               "ob_grad_div_tiled: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(terms && faces && corner_offsets && corner_slots && tile_faces && tile_counts && corner_codes && u &&
                   out,
               "ob_grad_div_tiled: null pointer");
    if (int st = allow_tile_memory()) return st;
    grad_div_tiled_kernel<<<ceil_div(n_vertices, kTileVertices), 256, kTileSmem, stream>>>(
        terms, faces, corner_offsets, corner_slots, tile_faces, tile_counts, corner_codes, n_vertices, n_columns, u,
        u_stride, u_iperm, out, out_stride, out_iperm, out_pinned);
    OB_CHECK_LAUNCH("grad_div_tiled");
    return OB_OK;
}

int ob_shift_packed(const double* phi, int n_vertices, int stride, const int32_t* iperm,
                    const int32_t* vertex_offsets, int n_meshes, const int32_t* sources, int n_columns,
                    double* sums, double* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 1 && n_meshes >= 1 && n_columns >= 1 && stride >= n_columns && stride <= kThreads,
               "ob_shift_packed: bad size");
    OB_REQUIRE(phi && vertex_offsets && sources && sums && out, "ob_shift_packed: null pointer");
    // At most one partial chunk a mesh beyond the full ones.
    const long long chunk_bound = (long long)n_vertices / kPackedChunk + n_meshes;
    Scratch scratch(stream);
    int* chunk_first = scratch.take<int>((size_t)n_meshes + 1);
    int4* chunks = scratch.take<int4>((size_t)chunk_bound);
    double* partials = scratch.take<double>((size_t)chunk_bound * stride);
    if (int st = scratch.commit()) return st;
    packed_chunks_kernel<<<1, kThreads, 0, stream>>>(vertex_offsets, n_meshes, chunk_first, chunks);
    OB_CHECK_LAUNCH("shift_packed chunks");
    const int threads = (kThreads / stride) * stride;
    packed_partials_kernel<<<(unsigned)chunk_bound, threads, 0, stream>>>(phi, stride, iperm, chunk_first, n_meshes,
                                                                        chunks, partials);
    OB_CHECK_LAUNCH("shift_packed partials");
    packed_fold_kernel<<<n_meshes, 32, 0, stream>>>(phi, stride, iperm, vertex_offsets, sources, n_columns,
                                                    chunk_first, partials, reinterpret_cast<double2*>(sums));
    OB_CHECK_LAUNCH("shift_packed fold");
    shift_packed_out_kernel<<<dim3(ceil_div(n_vertices, 32), ceil_div(n_columns, 32)), dim3(32, 8), 0, stream>>>(
        phi, n_vertices, stride, iperm, vertex_offsets, n_meshes, sources, n_columns,
        reinterpret_cast<const double2*>(sums), out);
    OB_CHECK_LAUNCH("shift_packed_out");
    return OB_OK;
}

int ob_seed_permuted(const int32_t* sources, const int32_t* source_offsets, int n_columns,
                     int n_vertices, const int32_t* iperm, const char* pinned, int stride,
                     double* rhs, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_columns >= 1 && stride >= n_columns && n_vertices >= 0, "ob_seed_permuted: bad size");
    OB_REQUIRE(sources && source_offsets && iperm && pinned && rhs, "ob_seed_permuted: null pointer");
    OB_CUDA(cudaMemsetAsync(rhs, 0, sizeof(double) * (size_t)n_vertices * stride, stream));
    seed_permuted_kernel<<<dim3(1, n_columns), 128, 0, stream>>>(sources, source_offsets, n_columns,
                                                               iperm, pinned, stride, rhs);
    OB_CHECK_LAUNCH("seed_permuted");
    return OB_OK;
}

int ob_shift_permuted(const double* phi, int n_vertices, int stride, const int32_t* iperm,
                      const int32_t* sources, const int32_t* source_offsets, int n_columns,
                      int orient, double* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 1 && n_columns >= 1 && stride >= n_columns, "ob_shift_permuted: bad size");
    OB_REQUIRE(phi && iperm && sources && source_offsets && out, "ob_shift_permuted: null pointer");
    OB_REQUIRE(stride <= kThreads, "ob_shift_permuted: stride above %d", kThreads);
    const int threads = (kThreads / stride) * stride;
    const long long total = (long long)n_vertices * stride;
    const int blocks = (int)std::max(1LL, std::min((total + threads * 16 - 1) / (threads * 16),
                                                   (long long)2 * sm_count()));
    Scratch scratch(stream);
    double* partials = scratch.take<double>((size_t)blocks * stride);
    double2* sums = scratch.take<double2>(n_columns);
    unsigned int* counter = scratch.take<unsigned int>(1);
    int st = scratch.commit();
    if (st) return st;
    OB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned int), stream));
    shift_sums_kernel<<<blocks, threads, 0, stream>>>(phi, n_vertices, stride, iperm, sources,
                                                       source_offsets, n_columns, orient, partials,
                                                       counter, sums);
    OB_CHECK_LAUNCH("shift_sums");
    shift_out_kernel<<<dim3(ceil_div(n_vertices, 32), ceil_div(n_columns, 32)), dim3(32, 8), 0,
                       stream>>>(phi, n_vertices, stride, iperm, sums, n_columns, out);
    OB_CHECK_LAUNCH("shift_out");
    return OB_OK;
}

}  // extern "C"
