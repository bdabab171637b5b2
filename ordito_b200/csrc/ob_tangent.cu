// f3: the vector heat method's tables and per-vertex steps on the device.
//
// Halfedge h = 3 f + k runs faces[3 f + k] -> faces[3 f + (k + 1) % 3] (ordito/kernels/halfedge.py:
// 41-114). Twins come from the operator pattern's sorted key runs (each run lists the corners whose
// opposite edge is one vertex pair), the rings from a walk over twin(prev(h)) (ordito/halfedge.py:
// 284-452, kernels/halfedge.py:656-752), then the tangent-space tables of ordito/tangent_space.py
// (polar angles, frames, transport rotations; kernels/tangent_space.py), the vector heat system's
// rows (kernels/heat.py:243-296, kernels/laplacian.py:1430-1465) expanded to a real 2n x 2n CSR
// whose rows 2v and 2v + 1 are vertex v's two tangent components, and the per-vertex tails of
// transport_tangent_vectors and log_map (kernels/heat.py:3881-4243).
//
// Every per-vertex gather reads its ring or its corners in a fixed order, so every result repeats
// bit for bit (no atomics on values).
#include <cfloat>
#include <algorithm>
#include <cmath>

#include "ob_geometry.cuh"
#include "ob_internal.cuh"

namespace ob {
namespace {

constexpr int kThreads = 256;
constexpr double kPi = 3.14159265358979323846;
constexpr float kMerge = 1e-8f;     // ordito/constants.py:13 (TOLERANCE_MERGE, float32)
constexpr float kZeroTol = 1e-12f;  // ordito/constants.py:15 (TOLERANCE_ZERO, float32)

struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 widen(f3 a) { return d3{(double)a.x, (double)a.y, (double)a.z}; }
__device__ __forceinline__ d3 sub(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 neg(d3 a) { return d3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross(d3 a, d3 b) {
    return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double length(d3 a) { return sqrt(dot(a, a)); }
__device__ __forceinline__ f3 scale(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }

__device__ __forceinline__ int prev_halfedge(int h) { return h - h % 3 + (h + 2) % 3; }
__device__ __forceinline__ int next_halfedge(int h) { return h - h % 3 + (h + 1) % 3; }

__device__ __forceinline__ int pattern_run_end(const unsigned long long* __restrict__ keys, int start, int count) {
    const unsigned long long key = keys[start];
    int p = start + 1;
    while (p < count && keys[p] == key) ++p;
    return p;
}

// Unsigned angle atan2(|a x b|, a . b) (kernels/predicates.py:458-472), in each precision.
__device__ __forceinline__ float vector_angle(f3 a, f3 b) { return atan2f(length(cross(a, b)), dot(a, b)); }
__device__ __forceinline__ double vector_angle(d3 a, d3 b) { return atan2(length(cross(a, b)), dot(a, b)); }

// A face's corner angles from its edges v1 - v0, v2 - v0, v2 - v1: two angles and pi less both,
// all zero when any is below the merge tolerance (kernels/triangles.py:427-439).
__device__ __forceinline__ void corner_angles(f3 e01, f3 e02, f3 e12, float* a) {
    a[0] = vector_angle(e01, e02);
    a[1] = vector_angle(neg(e01), e12);
    a[2] = (float)kPi - a[0] - a[1];
    if (a[0] < kMerge || a[1] < kMerge || a[2] < kMerge) a[0] = a[1] = a[2] = 0.0f;
}
__device__ __forceinline__ void corner_angles(d3 e01, d3 e02, d3 e12, double* a) {
    a[0] = vector_angle(e01, e02);
    a[1] = vector_angle(neg(e01), e12);
    a[2] = kPi - a[0] - a[1];
    const double tol = (double)kMerge;
    if (a[0] < tol || a[1] < tol || a[2] < tol) a[0] = a[1] = a[2] = 0.0;
}

// The float32 interior angle at the corner halfedge h leaves (kernels/triangles.py:486-493).
__device__ __forceinline__ float halfedge_corner_angle(const float* __restrict__ xyz, const int* __restrict__ faces,
                                                      int h) {
    const int f = h / 3;
    const f3 v0 = load_f3(xyz, faces[3 * f]), v1 = load_f3(xyz, faces[3 * f + 1]),
             v2 = load_f3(xyz, faces[3 * f + 2]);
    float a[3];
    corner_angles(sub(v1, v0), sub(v2, v0), sub(v2, v1), a);
    return a[h % 3];
}

// ring_tangent_scale (kernels/tangent_space.py:32-45): 2 pi / total (pi at a rim), 0 for no angle.
template <typename T>
__device__ __forceinline__ T ring_scale(T total, bool boundary) {
    if (total > (T)kZeroTol) return (boundary ? (T)kPi : (T)(2.0 * kPi)) / total;
    return (T)0;
}

// The slot polar angle 0 is measured from: an open fan's first (its outgoing boundary halfedge),
// else the slot of the ring's largest halfedge, its highest-index face's (kernels/tangent_space.py:
// 48-61).
__device__ __forceinline__ int reference_slot(const int* __restrict__ ring, int begin, int end, bool boundary) {
    int best = begin;
    if (!boundary)
        for (int j = begin + 1; j < end; ++j)
            if (ring[j] > ring[best]) best = j;
    return best - begin;
}

// ---------------------------------------------------------------------------------------------
// Halfedge tables.
// ---------------------------------------------------------------------------------------------

// One thread per upper pattern entry (i < j): its run lists the corners whose opposite edge is
// {i, j}; their opposite halfedges are the edge's halfedges (ordito/halfedge.py:59-172).
__global__ void twins_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                             const int* __restrict__ run_start, const unsigned long long* __restrict__ keys,
                             int n_keys, const int* __restrict__ order, const int* __restrict__ faces, int n_vertices,
                             int* __restrict__ twins, int* __restrict__ defects) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_vertices) return;
    for (int k = offsets[i]; k < offsets[i + 1]; ++k) {
        if (columns[k] <= i) continue;
        const int s = run_start[k], e = pattern_run_end(keys, s, n_keys);
        if (e - s > 2) {
            atomicAdd(defects, 1);
            continue;
        }
        if (e - s < 2) continue;  // a boundary edge: its halfedge keeps -1
        const int qa = order[s], qb = order[s + 1];
        const int ha = 3 * (qa / 3) + (qa % 3 + 1) % 3, hb = 3 * (qb / 3) + (qb % 3 + 1) % 3;
        if (faces[ha] == faces[hb]) {
            atomicAdd(defects + 1, 1);
            continue;
        }
        twins[ha] = hb;
        twins[hb] = ha;
    }
}

// One thread per vertex: its ring from its outgoing boundary halfedge (the lowest-indexed one),
// else from its lowest-indexed outgoing halfedge, walked by twin(prev(h)) and bounded by its
// degree; a walk that closes early (a pinched vertex) counts into defects[0] and leaves -1 in its
// remaining slots (kernels/halfedge.py:656-752). The corner index lists a vertex's corners, which
// are its outgoing halfedges, in ascending order.
__global__ void rings_kernel(const int* __restrict__ corner_offsets, const int* __restrict__ corner_slots,
                             const int* __restrict__ twins, int n_vertices, int* __restrict__ ring,
                             unsigned char* __restrict__ is_boundary, int* __restrict__ defects) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_vertices) return;
    const int begin = corner_offsets[v], degree = corner_offsets[v + 1] - begin;
    if (degree == 0) {
        is_boundary[v] = 0;
        return;
    }
    int start = corner_slots[begin];
    bool boundary = false;
    for (int j = begin; j < begin + degree; ++j)
        if (twins[corner_slots[j]] < 0) {
            start = corner_slots[j];
            boundary = true;
            break;
        }
    is_boundary[v] = boundary ? 1 : 0;
    int count = 0, h = start;
    while (count < degree) {
        ring[begin + count] = h;
        ++count;
        const int nxt = twins[prev_halfedge(h)];
        if (nxt < 0 || nxt == start) break;
        h = nxt;
    }
    if (count != degree) {
        atomicAdd(defects, 1);
        for (int j = begin + count; j < begin + degree; ++j) ring[j] = -1;
    }
}

// ---------------------------------------------------------------------------------------------
// Tangent spaces (ordito/tangent_space.py, kernels/tangent_space.py).
// ---------------------------------------------------------------------------------------------

// A face's three float64 corner angles from its float32 corners widened (kernels/triangles.py:
// 476-482, park_corner_angles at kernels/tangent_space.py:275-295).
__global__ void corner_angles_kernel(const float* __restrict__ xyz, const int* __restrict__ faces, int n_faces,
                                     double* __restrict__ angles) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const d3 v0 = widen(load_f3(xyz, faces[3 * f])), v1 = widen(load_f3(xyz, faces[3 * f + 1])),
             v2 = widen(load_f3(xyz, faces[3 * f + 2]));
    double a[3];
    corner_angles(sub(v1, v0), sub(v2, v0), sub(v2, v1), a);
    angles[3 * f] = a[0];
    angles[3 * f + 1] = a[1];
    angles[3 * f + 2] = a[2];
}

// A caller's float32 corner-angle table widened (kernels/tangent_space.py:63-70).
__global__ void widen_angles_kernel(const float* __restrict__ face_angles, long long count, double* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < count) out[i] = (double)face_angles[i];
}

// A tangent vector (a, b) in a vertex's frame as a * basis_x + b * basis_y (kernels/heat.py:583-596).
__global__ void tangent_to_world_kernel(const float* __restrict__ tangent, const float* __restrict__ basis_x,
                                        const float* __restrict__ basis_y, int n, float* __restrict__ out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const float a = tangent[2 * v], b = tangent[2 * v + 1];
    const f3 w = add(scale(load_f3(basis_x, v), a), scale(load_f3(basis_y, v), b));
    out[3 * v] = w.x;
    out[3 * v + 1] = w.y;
    out[3 * v + 2] = w.z;
}

// A caller's transport angles as rotations (cos, sin) (ordito/heat.py:1958, predicates.py:686).
__global__ void polar_unit_kernel(const double* __restrict__ angles, int n, double* __restrict__ out) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n) return;
    out[2 * h] = cos(angles[h]);
    out[2 * h + 1] = sin(angles[h]);
}

// One thread per vertex: the corner angles summed in ring order, rescaled to a full turn (half at
// a rim), laid out from the reference slot (kernels/tangent_space.py:102-133).
__global__ void tangent_angles_kernel(const int* __restrict__ ring_offsets, const int* __restrict__ ring,
                                      const unsigned char* __restrict__ is_boundary,
                                      const double* __restrict__ corner, int n_vertices, int n_halfedges,
                                      double* __restrict__ out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_vertices) return;
    const int begin = ring_offsets[v], end = ring_offsets[v + 1], n = end - begin;
    if (n <= 0) return;
    double total = 0.0;
    for (int j = begin; j < end; ++j)
        if (ring[j] >= 0 && ring[j] < n_halfedges) total += corner[ring[j]];
    const bool boundary = is_boundary[v] != 0;
    const double s = ring_scale(total, boundary);
    const int start = reference_slot(ring, begin, end, boundary);
    double acc = 0.0;
    for (int t = 0; t < n; ++t) {
        const int h = ring[begin + (start + t) % n];
        if (h < 0 || h >= n_halfedges) continue;  // a pinched vertex's unfilled slot
        out[h] = s * acc;
        acc += corner[h];
    }
}

__device__ __forceinline__ f3 normalize(f3 a) {
    const float l = length(a);
    return l > 0.0f ? f3{a.x / l, a.y / l, a.z / l} : f3{0.0f, 0.0f, 0.0f};
}

// kernels/predicates.py:163-182: the normal crossed with x, or with y where x is the nearer.
__device__ __forceinline__ f3 any_perpendicular(f3 n) {
    const f3 axis = fabsf(n.x) > fabsf(n.y) ? f3{0.0f, 1.0f, 0.0f} : f3{1.0f, 0.0f, 0.0f};
    return normalize(cross(n, axis));
}

// One thread per vertex: the angle-weighted normal gathered over the ring (float32 terms widened
// into a float64 sum; kernels/normals.py:52-169) and the frame whose basis_x is polar angle 0
// fitted to the whole fan (kernels/tangent_space.py:335-480).
__global__ void frames_kernel(const float* __restrict__ xyz, const int* __restrict__ faces,
                              const int* __restrict__ ring_offsets, const int* __restrict__ ring,
                              const unsigned char* __restrict__ is_boundary, int n_vertices, int n_halfedges,
                              const float* __restrict__ given_normals, float* __restrict__ basis_x,
                              float* __restrict__ basis_y, float* __restrict__ normals) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_vertices) return;
    const int begin = ring_offsets[v], end = ring_offsets[v + 1], n = end - begin;
    const bool boundary = is_boundary[v] != 0;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    float angle_total = 0.0f;
    for (int j = begin; j < end; ++j) {
        const int h = ring[j], f = h / 3;
        if (h < 0 || h >= n_halfedges) continue;  // a pinched vertex's unfilled slot
        f3 fn;
        float area;
        normal_and_area(load_f3(xyz, faces[3 * f]), load_f3(xyz, faces[3 * f + 1]), load_f3(xyz, faces[3 * f + 2]),
                        &fn, &area);
        const float angle = halfedge_corner_angle(xyz, faces, h);
        const f3 term = scale(fn, angle);
        sx += (double)term.x;
        sy += (double)term.y;
        sz += (double)term.z;
        angle_total += angle;
    }
    f3 normal;
    if (given_normals != nullptr) {
        // A caller's normals (kernels/tangent_space.py:551-553): read, not written.
        normal = load_f3(given_normals, v);
    } else {
        const double nl = sqrt(sx * sx + sy * sy + sz * sz);
        if (nl > 0.0) {
            sx /= nl;
            sy /= nl;
            sz /= nl;
        }
        normal = f3{(float)sx, (float)sy, (float)sz};
        normals[3 * v] = normal.x;
        normals[3 * v + 1] = normal.y;
        normals[3 * v + 2] = normal.z;
    }
    f3 bx;
    if (length(normal) <= kZeroTol) {
        bx = f3{1.0f, 0.0f, 0.0f};
        basis_x[3 * v] = 1.0f, basis_x[3 * v + 1] = 0.0f, basis_x[3 * v + 2] = 0.0f;
        basis_y[3 * v] = 0.0f, basis_y[3 * v + 1] = 1.0f, basis_y[3 * v + 2] = 0.0f;
        return;
    }
    const int href = n > 0 ? ring[begin + reference_slot(ring, begin, end, boundary)] : -1;
    if (href < 0 || href >= n_halfedges) {
        bx = any_perpendicular(normal);
    } else {
        const int start = reference_slot(ring, begin, end, boundary);
        const f3 origin = load_f3(xyz, v);
        const f3 direction = sub(load_f3(xyz, faces[next_halfedge(href)]), origin);
        const f3 tangential = sub(direction, scale(normal, dot(direction, normal)));
        const float ref_length = length(tangential);
        bx = any_perpendicular(normal);
        if (ref_length > kZeroTol)
            bx = f3{tangential.x / ref_length, tangential.y / ref_length, tangential.z / ref_length};
        const float s = ring_scale(angle_total, boundary);
        if (s > 0.0f) {
            const f3 fy = cross(normal, bx);
            float ax = 0.0f, ay = 0.0f, acc = 0.0f;
            for (int t = 0; t < n; ++t) {
                const int h = ring[begin + (start + t) % n];
                if (h < 0 || h >= n_halfedges) continue;
                const f3 edge = sub(load_f3(xyz, faces[next_halfedge(h)]), origin);
                const float e0 = dot(edge, bx), e1 = dot(edge, fy);
                const float theta = s * acc;
                const float c = cosf(theta), sn = sinf(theta);
                ax += e0 * c + e1 * sn;
                ay += e1 * c - e0 * sn;
                acc += halfedge_corner_angle(xyz, faces, h);
            }
            if (boundary && ring[end - 1] >= 0 && ring[end - 1] < n_halfedges) {
                const f3 rim = sub(load_f3(xyz, faces[prev_halfedge(ring[end - 1])]), origin);
                ax -= dot(rim, bx);
                ay -= dot(rim, fy);
            }
            if (sqrtf(ax * ax + ay * ay) > kZeroTol * ref_length) bx = normalize(add(scale(bx, ax), scale(fy, ay)));
        }
    }
    const f3 by = cross(normal, bx);
    basis_x[3 * v] = bx.x, basis_x[3 * v + 1] = bx.y, basis_x[3 * v + 2] = bx.z;
    basis_y[3 * v] = by.x, basis_y[3 * v + 1] = by.y, basis_y[3 * v + 2] = by.z;
}

// One thread per halfedge: rho = wrap(theta_twin + pi - theta_h), pi standing in for a boundary
// edge's missing twin, and its rotation (cos, sin) (kernels/tangent_space.py:700-730).
__global__ void transport_kernel(const int* __restrict__ twins, const double* __restrict__ tangent, int n_halfedges,
                                 double* __restrict__ rho, double* __restrict__ rotations) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n_halfedges) return;
    const int twin = twins[h];
    const double opposite = twin >= 0 ? tangent[twin] : kPi;
    const double a = opposite + kPi - tangent[h];
    const double r = atan2(sin(a), cos(a));
    if (rho) rho[h] = r;
    if (rotations) {
        rotations[2 * h] = cos(r);
        rotations[2 * h + 1] = sin(r);
    }
}

// ---------------------------------------------------------------------------------------------
// The vector heat system.
// ---------------------------------------------------------------------------------------------

// Half-cotangents from the float32 corners widened to float64 (kernels/laplacian.py:94-136).
__global__ void half_cot_f64_kernel(const float* __restrict__ xyz, const int* __restrict__ faces, int n_faces,
                                    double* __restrict__ cot) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const d3 v0 = widen(load_f3(xyz, faces[3 * f])), v1 = widen(load_f3(xyz, faces[3 * f + 1])),
             v2 = widen(load_f3(xyz, faces[3 * f + 2]));
    // Twice the area at the corner opposite the longest edge (kernels/predicates.py:106-130).
    const d3 ab = sub(v1, v0), bc = sub(v2, v1), ca = sub(v0, v2);
    const double l_ab = dot(ab, ab), l_bc = dot(bc, bc), l_ca = dot(ca, ca);
    d3 area_vector;
    if (l_bc >= l_ca && l_bc >= l_ab)
        area_vector = cross(ab, neg(ca));
    else if (l_ca >= l_ab)
        area_vector = cross(bc, neg(ab));
    else
        area_vector = cross(ca, neg(bc));
    const double den = 2.0 * length(area_vector);
    if (den <= 0.0) {
        cot[3 * f] = cot[3 * f + 1] = cot[3 * f + 2] = 0.0;
        return;
    }
    cot[3 * f] = dot(sub(v1, v0), sub(v2, v0)) / den;
    cot[3 * f + 1] = dot(sub(v2, v1), sub(v0, v1)) / den;
    cot[3 * f + 2] = dot(sub(v0, v2), sub(v1, v2)) / den;
}

// The expanded pattern: pattern row i of length m becomes rows 2i and 2i + 1 of length 2m, entry
// k's block at columns 2c, 2c + 1 (ascending, as the pattern's columns are).
__global__ void block_pattern_kernel(const int* __restrict__ offsets, const int* __restrict__ columns, int n,
                                     int* __restrict__ block_offsets, int* __restrict__ block_columns) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) {
        block_offsets[2 * n] = 4 * offsets[n];
        return;
    }
    const int start = offsets[i], m = offsets[i + 1] - start;
    block_offsets[2 * i] = 4 * start;
    block_offsets[2 * i + 1] = 4 * start + 2 * m;
    for (int a = 0; a < 2; ++a) {
        int* out = block_columns + 4 * start + a * 2 * m;
        for (int j = 0; j < m; ++j) {
            out[2 * j] = 2 * columns[start + j];
            out[2 * j + 1] = 2 * columns[start + j] + 1;
        }
    }
}

// One thread per pattern row: M + factor L_connection over the expanded pattern. An off-diagonal
// block is factor * sum -w R(+-rho) over the edge's corners in sorted (face) order, the sine
// negated when the halfedge leaves this row's vertex; the diagonal block is (factor * sum w + m) I
// (kernels/heat.py:243-296, kernels/laplacian.py:1430-1465, kernels/linalg.py:1594-1633).
__global__ void vector_rows_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                                   const int* __restrict__ run_start, const unsigned long long* __restrict__ keys,
                                   int n_keys, const int* __restrict__ order, int n, const int* __restrict__ faces,
                                   const double* __restrict__ cot, const double* __restrict__ rotations,
                                   const double* __restrict__ mass, double scale, const double* __restrict__ edge_sums,
                                   int from_edges, double* __restrict__ values) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double factor = scale;
    if (from_edges) {
        double h = 0.0;
        if (edge_sums[1] > 0.0) h = edge_sums[0] / edge_sums[1];
        factor = scale * (h * h);
    }
    const int start = offsets[i], m = offsets[i + 1] - start;
    double* row0 = values + 4 * (size_t)start;
    double* row1 = row0 + 2 * m;
    double weight = 0.0;
    int slot = -1;
    for (int j = 0; j < m; ++j) {
        const int k = start + j;
        if (columns[k] == i) {
            slot = j;
            continue;
        }
        double b00 = 0.0, b01 = 0.0, b10 = 0.0, b11 = 0.0;
        const int s = run_start[k], e = pattern_run_end(keys, s, n_keys);
        for (int p = s; p < e; ++p) {
            const int q = order[p];
            const int h = 3 * (q / 3) + (q % 3 + 1) % 3;
            const double w = cot[q];
            const double c = rotations[2 * h];
            const double sine = faces[h] == i ? -rotations[2 * h + 1] : rotations[2 * h + 1];
            b00 += -w * c;
            b01 += -w * -sine;
            b10 += -w * sine;
            b11 += -w * c;
            weight += w;
        }
        row0[2 * j] = factor * b00;
        row0[2 * j + 1] = factor * b01;
        row1[2 * j] = factor * b10;
        row1[2 * j + 1] = factor * b11;
    }
    if (slot >= 0) {
        const double d = factor * weight + mass[i];
        row0[2 * slot] = d;
        row0[2 * slot + 1] = 0.0;
        row1[2 * slot] = 0.0;
        row1[2 * slot + 1] = d;
    }
}

// ---------------------------------------------------------------------------------------------
// transport_tangent_vectors (kernels/heat.py:3881-3901, :3975-3996).
// ---------------------------------------------------------------------------------------------

__global__ void transport_seed_kernel(const int* __restrict__ sources, const float* __restrict__ vectors, int k, int n,
                                      double* __restrict__ field, double* __restrict__ scalars,
                                      int* __restrict__ invalid) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= k) return;
    const int v = sources[s];
    if (v < 0 || v >= n) {
        *invalid = 1;
        return;
    }
    const double x = (double)vectors[2 * s], y = (double)vectors[2 * s + 1];
    atomicAdd(field + 2 * (size_t)v, x);
    atomicAdd(field + 2 * (size_t)v + 1, y);
    atomicAdd(scalars + 2 * (size_t)v, 1.0);
    atomicAdd(scalars + 2 * (size_t)v + 1, sqrt(x * x + y * y));
}

// normalize(v) and |v| without underflow: scaled by the largest component first
// (kernels/predicates.py:703-724).
__device__ __forceinline__ void stable_normalize2(double x, double y, double* ux, double* uy, double* len) {
    const double largest = fmax(fabs(x), fabs(y));
    if (largest == 0.0) {
        *ux = *uy = *len = 0.0;
        return;
    }
    const double a = x / largest, b = y / largest;
    const double l = sqrt(a * a + b * b);
    *ux = a / l;
    *uy = b / l;
    *len = largest * l;
}

__global__ void transport_tail_kernel(const double* __restrict__ field, const double* __restrict__ scalars, int n,
                                      double resolved_fraction, float* __restrict__ transported,
                                      unsigned char* __restrict__ resolved) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const double indicator = scalars[2 * (size_t)v], diffused_magnitude = scalars[2 * (size_t)v + 1];
    const double magnitude = indicator != 0.0 ? diffused_magnitude / indicator : 0.0;
    double ux, uy, len;
    stable_normalize2(field[2 * (size_t)v], field[2 * (size_t)v + 1], &ux, &uy, &len);
    transported[2 * v] = (float)(magnitude * ux);
    transported[2 * v + 1] = (float)(magnitude * uy);
    resolved[v] = len > resolved_fraction * diffused_magnitude ? 1 : 0;
}

// ---------------------------------------------------------------------------------------------
// log_map, method "heat_geodesic" (kernels/heat.py:3904-3916, :3999-4071).
// ---------------------------------------------------------------------------------------------

// Per face: its unit distance gradient (float64, scaled before normalising), narrowed and times
// the float32 area (kernels/heat.py:3999-4027, kernels/triangles.py:835-894).
__global__ void face_gradient_area_kernel(const float* __restrict__ xyz, const int* __restrict__ faces, int n_faces,
                                          const float* __restrict__ normals, const float* __restrict__ areas,
                                          const double* __restrict__ values, float* __restrict__ out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const int i0 = faces[3 * f], i1 = faces[3 * f + 1], i2 = faces[3 * f + 2];
    const d3 v0 = widen(load_f3(xyz, i0)), v1 = widen(load_f3(xyz, i1)), v2 = widen(load_f3(xyz, i2));
    const d3 nrm = widen(load_f3(normals, f));
    const float area32 = areas[f];
    const double area = (double)area32;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    if (area > 0.0) {
        const d3 c0 = cross(nrm, sub(v2, v1)), c1 = cross(nrm, sub(v0, v2)), c2 = cross(nrm, sub(v1, v0));
        const double u0 = values[i0], u1 = values[i1], u2 = values[i2];
        const double den = 2.0 * area;
        gx = (u0 * c0.x + u1 * c1.x + u2 * c2.x) / den;
        gy = (u0 * c0.y + u1 * c1.y + u2 * c2.y) / den;
        gz = (u0 * c0.z + u1 * c1.z + u2 * c2.z) / den;
    }
    const double largest = fmax(fabs(gx), fmax(fabs(gy), fabs(gz)));
    float x = 0.0f, y = 0.0f, z = 0.0f;
    if (largest > 0.0) {
        const double a = gx / largest, b = gy / largest, c = gz / largest;
        const double l = sqrt(a * a + b * b + c * c);
        x = (float)(a / l);
        y = (float)(b / l);
        z = (float)(c / l);
    }
    out[3 * f] = x * area32;
    out[3 * f + 1] = y * area32;
    out[3 * f + 2] = z * area32;
}

// Per vertex: its faces' values summed in ascending corner order (the deterministic corner sum,
// kernels/scatter.py:801-819), float32 for a vec3 field, float64 for a scalar one.
__global__ void gather_corners_vec3_kernel(const float* __restrict__ face_values, const int* __restrict__ corner_offsets,
                                           const int* __restrict__ corner_slots, int n, float* __restrict__ out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    float x = 0.0f, y = 0.0f, z = 0.0f;
    for (int j = corner_offsets[v]; j < corner_offsets[v + 1]; ++j) {
        const int f = corner_slots[j] / 3;
        x += face_values[3 * f];
        y += face_values[3 * f + 1];
        z += face_values[3 * f + 2];
    }
    out[3 * v] = x;
    out[3 * v + 1] = y;
    out[3 * v + 2] = z;
}

__global__ void gather_corners_scalar_kernel(const double* __restrict__ corner_values,
                                             const int* __restrict__ corner_offsets,
                                             const int* __restrict__ corner_slots, int n, double* __restrict__ out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    double sum = 0.0;
    for (int j = corner_offsets[v]; j < corner_offsets[v + 1]; ++j) sum += corner_values[corner_slots[j]];
    out[v] = sum;
}

// Polar coordinates as seen from the source: the angle from the transported reference direction
// to the outward distance gradient, at the distance's radius; angle 0 where either direction
// vanished (kernels/heat.py:4030-4071).
__global__ void log_map_angles_kernel(const float* __restrict__ gradient, const float* __restrict__ basis_x,
                                      const float* __restrict__ basis_y, const double* __restrict__ transported,
                                      const double* __restrict__ distance, int n, float* __restrict__ out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    double ux, uy, len;
    stable_normalize2(transported[2 * (size_t)v], transported[2 * (size_t)v + 1], &ux, &uy, &len);
    const float rx = (float)ux, ry = (float)uy;
    const f3 g = load_f3(gradient, v);
    const float px = dot(g, load_f3(basis_x, v)), py = dot(g, load_f3(basis_y, v));
    float ox = 0.0f, oy = 0.0f;
    const float largest = fmaxf(fabsf(px), fabsf(py));
    if (largest != 0.0f) {
        const float a = px / largest, b = py / largest;
        const float l = sqrtf(a * a + b * b);
        ox = a / l;
        oy = b / l;
    }
    const float r = (float)distance[v];
    if (sqrtf(rx * rx + ry * ry) <= kZeroTol || sqrtf(ox * ox + oy * oy) <= kZeroTol) {
        out[2 * v] = r;
        out[2 * v + 1] = 0.0f;
        return;
    }
    const float angle = atan2f(rx * oy - ry * ox, rx * ox + ry * oy);
    out[2 * v] = r * cosf(angle);
    out[2 * v + 1] = r * sinf(angle);
}

// ---------------------------------------------------------------------------------------------
// log_map, method "potpourri3d" (kernels/heat.py:4074-4243): two tangent fields as the columns of
// one [2n][2] block, column 0 the outward ball (radial), column 1 the reference direction.
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ void complex_add_product(double ax, double ay, double angle, double* out, size_t stride) {
    const double c = cos(angle), s = sin(angle);
    out[0] += ax * c - ay * s;
    out[stride] += ax * s + ay * c;
}

// One thread walks the source's ring in its fixed order (appendix A of the vector heat method).
__global__ void outward_ball_kernel(const float* __restrict__ xyz, const int* __restrict__ faces,
                                    const int* __restrict__ ring_offsets, const int* __restrict__ ring,
                                    const double* __restrict__ tangent, const double* __restrict__ transport,
                                    int source, double* __restrict__ rhs) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    rhs[4 * (size_t)source + 1] = 1.0;  // column 1 of row 2 source: the reference direction (1, 0)
    const d3 pa = widen(load_f3(xyz, source));
    for (int j = ring_offsets[source]; j < ring_offsets[source + 1]; ++j) {
        const int ab = ring[j], f = ab / 3, k = ab - 3 * f;
        if (ab < 0) continue;
        const int bc = 3 * f + (k + 1) % 3, ca = 3 * f + (k + 2) % 3;
        const int b = faces[bc], c = faces[ca];
        const d3 pb = widen(load_f3(xyz, b)), pc = widen(load_f3(xyz, c));
        const double twice_area = length(cross(sub(pb, pa), sub(pc, pa)));
        if (twice_area == 0.0) continue;
        const double theta = vector_angle(sub(pb, pa), sub(pc, pa));
        const double gamma = vector_angle(sub(pa, pb), sub(pc, pb));
        const double sine = sin(theta);
        const double swing = theta * cos(theta) - sine;
        const double height_b = twice_area / length(sub(pc, pa));
        complex_add_product(-theta * sine / (2.0 * height_b), swing / (2.0 * height_b),
                            tangent[ab] + transport[ab] - kPi, rhs + 4 * (size_t)b, 2);
        const double height_c = twice_area / length(sub(pb, pa));
        complex_add_product(-theta * sine / (2.0 * height_c), -swing / (2.0 * height_c), tangent[ca],
                            rhs + 4 * (size_t)c, 2);
        const double height_a = twice_area / length(sub(pc, pb));
        const double alpha = 0.5 * kPi - gamma;
        const double ax = -(theta * cos(alpha) + cos(alpha - theta) * sine) / (2.0 * height_a);
        const double ay = -(cos(alpha) - cos(alpha - 2.0 * theta) + 2.0 * theta * sin(alpha)) / (4.0 * height_a);
        complex_add_product(ax, ay, tangent[ab], rhs + 4 * (size_t)source, 2);
    }
}

__device__ __forceinline__ void unit_radial(const double* __restrict__ fields, int v, int source, double* x,
                                            double* y) {
    if (v == source) {
        *x = *y = 0.0;
        return;
    }
    double len;
    stable_normalize2(fields[4 * (size_t)v], fields[4 * (size_t)v + 2], x, y, &len);
}

// One face's flux of the unit radial field along its halfedge h = i -> j (kernels/heat.py:
// 4163-4190).
__device__ __forceinline__ double radial_flux(const float* __restrict__ xyz, const int* __restrict__ faces,
                                              const double* __restrict__ tangent,
                                              const double* __restrict__ transport,
                                              const double* __restrict__ fields, int source, double w, int h, int nh) {
    const int i = faces[h], j = faces[nh];
    double rix, riy, rjx, rjy;
    unit_radial(fields, i, source, &rix, &riy);
    unit_radial(fields, j, source, &rjx, &rjy);
    const double c = cos(-transport[h]), s = sin(-transport[h]);
    const double bx = rjx * c - rjy * s, by = rjx * s + rjy * c;
    const double len = length(sub(widen(load_f3(xyz, j)), widen(load_f3(xyz, i))));
    const double ex = len * cos(tangent[h]), ey = len * sin(tangent[h]);
    return w * ((0.5 * (rix + bx)) * ex + (0.5 * (riy + by)) * ey);
}

__global__ void radial_divergence_kernel(const float* __restrict__ xyz, const int* __restrict__ faces, int n_faces,
                                         const double* __restrict__ tangent, const double* __restrict__ transport,
                                         const double* __restrict__ fields, int source, const float* __restrict__ cot,
                                         double* __restrict__ corner) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces) return;
    const int base = 3 * f;
    const double f01 = radial_flux(xyz, faces, tangent, transport, fields, source, (double)cot[base + 2], base, base + 1);
    const double f12 = radial_flux(xyz, faces, tangent, transport, fields, source, (double)cot[base], base + 1, base + 2);
    const double f20 = radial_flux(xyz, faces, tangent, transport, fields, source, (double)cot[base + 1], base + 2, base);
    corner[base] = f20 - f01;
    corner[base + 1] = f01 - f12;
    corner[base + 2] = f12 - f20;
}

// The radial direction measured from the transported reference, radial * conj(horizontal), at the
// distance from the source (kernels/heat.py:4228-4243).
__global__ void log_map_fields_kernel(const double* __restrict__ fields, const double* __restrict__ distance,
                                      int source, int n, float* __restrict__ out) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    double rx, ry, hx, hy, len;
    unit_radial(fields, v, source, &rx, &ry);
    stable_normalize2(fields[4 * (size_t)v + 1], fields[4 * (size_t)v + 3], &hx, &hy, &len);
    const double d = distance[v] - distance[source];
    out[2 * v] = (float)(d * (rx * hx + ry * hy));
    out[2 * v + 1] = (float)(d * (ry * hx - rx * hy));
}

inline int blocks_for(long long n) { return std::max(1, ceil_div(n, kThreads)); }

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_halfedge_twins(const int32_t* offsets, const int32_t* columns, const int32_t* run_start, const uint64_t* keys,
                      int n_keys, const int32_t* order, const int32_t* faces, int n_faces, int n_vertices,
                      int32_t* twins, int32_t* defects, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 0 && n_vertices >= 0, "ob_halfedge_twins: bad size");
    OB_REQUIRE(defects != nullptr, "ob_halfedge_twins: null defects");
    OB_CUDA(cudaMemsetAsync(defects, 0, 2 * sizeof(int32_t), stream));
    if (n_faces == 0) return OB_OK;
    OB_REQUIRE(offsets && columns && run_start && keys && order && faces && twins, "ob_halfedge_twins: null pointer");
    OB_CUDA(cudaMemsetAsync(twins, 0xFF, sizeof(int32_t) * 3 * (size_t)n_faces, stream));
    if (n_vertices == 0) return OB_OK;
    twins_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), n_keys, order, faces,
        n_vertices, twins, defects);
    OB_CHECK_LAUNCH("halfedge twins");
    return OB_OK;
}

int ob_vertex_one_rings(const int32_t* corner_offsets, const int32_t* corner_slots, const int32_t* twins,
                        int n_vertices, int32_t* ring_halfedges, uint8_t* is_boundary, int32_t* defects,
                        ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && defects, "ob_vertex_one_rings: bad argument");
    OB_CUDA(cudaMemsetAsync(defects, 0, sizeof(int32_t), stream));
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(corner_offsets && corner_slots && twins && ring_halfedges && is_boundary,
               "ob_vertex_one_rings: null pointer");
    rings_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(corner_offsets, corner_slots, twins, n_vertices,
                                                                  ring_halfedges, is_boundary, defects);
    OB_CHECK_LAUNCH("vertex one rings");
    return OB_OK;
}

int ob_halfedge_tangent_angles(const float* xyz, const int32_t* faces, int n_faces, int n_vertices,
                               const int32_t* ring_offsets, const int32_t* ring_halfedges, const uint8_t* is_boundary,
                               const float* face_angles, double* corner_angles, double* angles,
                               ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 0 && n_vertices >= 0, "ob_halfedge_tangent_angles: bad size");
    if (n_faces == 0) return OB_OK;
    OB_REQUIRE(ring_offsets && ring_halfedges && is_boundary && corner_angles && angles &&
                   (face_angles || (xyz && faces)),
               "ob_halfedge_tangent_angles: null pointer");
    OB_CUDA(cudaMemsetAsync(angles, 0, sizeof(double) * 3 * (size_t)n_faces, stream));
    if (face_angles != nullptr) {
        widen_angles_kernel<<<blocks_for(3LL * n_faces), kThreads, 0, stream>>>(face_angles, 3LL * n_faces,
                                                                                corner_angles);
    } else {
        corner_angles_kernel<<<blocks_for(n_faces), kThreads, 0, stream>>>(xyz, faces, n_faces, corner_angles);
    }
    OB_CHECK_LAUNCH("corner angles");
    if (n_vertices == 0) return OB_OK;
    tangent_angles_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(ring_offsets, ring_halfedges, is_boundary,
                                                                           corner_angles, n_vertices, 3 * n_faces,
                                                                           angles);
    OB_CHECK_LAUNCH("tangent angles");
    return OB_OK;
}

int ob_vertex_tangent_frames(const float* xyz, const int32_t* faces, int n_faces, int n_vertices,
                             const int32_t* ring_offsets, const int32_t* ring_halfedges, const uint8_t* is_boundary,
                             const float* given_normals, float* basis_x, float* basis_y, float* normals,
                             ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0, "ob_vertex_tangent_frames: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(xyz && ring_offsets && is_boundary && basis_x && basis_y && (normals || given_normals),
               "ob_vertex_tangent_frames: null pointer");
    frames_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(xyz, faces, ring_offsets, ring_halfedges,
                                                                   is_boundary, n_vertices, 3 * n_faces, given_normals,
                                                                   basis_x, basis_y, normals);
    OB_CHECK_LAUNCH("vertex tangent frames");
    return OB_OK;
}

int ob_halfedge_transport(const int32_t* twins, const double* tangent_angles, int n_halfedges, double* rho,
                          double* rotations, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_halfedges >= 0, "ob_halfedge_transport: bad size");
    if (n_halfedges == 0) return OB_OK;
    OB_REQUIRE(twins && tangent_angles && (rho || rotations), "ob_halfedge_transport: null pointer");
    transport_kernel<<<blocks_for(n_halfedges), kThreads, 0, stream>>>(twins, tangent_angles, n_halfedges, rho,
                                                                       rotations);
    OB_CHECK_LAUNCH("halfedge transport");
    return OB_OK;
}

int ob_polar_unit(const double* angles, int n, double* rotations, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n >= 0, "ob_polar_unit: bad size");
    if (n == 0) return OB_OK;
    OB_REQUIRE(angles && rotations, "ob_polar_unit: null pointer");
    polar_unit_kernel<<<blocks_for(n), kThreads, 0, stream>>>(angles, n, rotations);
    OB_CHECK_LAUNCH("polar unit");
    return OB_OK;
}

int ob_half_cot_f64(const float* xyz, const int32_t* faces, int n_faces, double* cot, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 0, "ob_half_cot_f64: bad size");
    if (n_faces == 0) return OB_OK;
    OB_REQUIRE(xyz && faces && cot, "ob_half_cot_f64: null pointer");
    half_cot_f64_kernel<<<blocks_for(n_faces), kThreads, 0, stream>>>(xyz, faces, n_faces, cot);
    OB_CHECK_LAUNCH("half cot f64");
    return OB_OK;
}

int ob_block_pattern(const int32_t* offsets, const int32_t* columns, int n_vertices, int32_t* block_offsets,
                     int32_t* block_columns, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && offsets && block_offsets, "ob_block_pattern: bad argument");
    OB_REQUIRE(n_vertices == 0 || (columns && block_columns), "ob_block_pattern: null pointer");
    block_pattern_kernel<<<blocks_for(n_vertices + 1), kThreads, 0, stream>>>(offsets, columns, n_vertices,
                                                                              block_offsets, block_columns);
    OB_CHECK_LAUNCH("block pattern");
    return OB_OK;
}

int ob_vector_heat_rows(const int32_t* offsets, const int32_t* columns, const int32_t* run_start, const uint64_t* keys,
                        int n_keys, const int32_t* order, int n_vertices, const int32_t* faces, const double* cot,
                        const double* rotations, const double* mass, double scale, const double* edge_sums,
                        int from_edges, double* values, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0, "ob_vector_heat_rows: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(offsets && columns && run_start && keys && order && faces && cot && rotations && mass && values,
               "ob_vector_heat_rows: null pointer");
    OB_REQUIRE(!from_edges || edge_sums != nullptr, "ob_vector_heat_rows: from_edges needs edge_sums");
    vector_rows_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), n_keys, order, n_vertices,
        faces, cot, rotations, mass, scale, edge_sums, from_edges, values);
    OB_CHECK_LAUNCH("vector heat rows");
    return OB_OK;
}

int ob_transport_seed(const int32_t* sources, const float* vectors, int n_sources, int n_vertices, double* field,
                      double* scalars, int32_t* invalid, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_sources >= 1 && n_vertices >= 1, "ob_transport_seed: bad size");
    OB_REQUIRE(sources && vectors && field && scalars && invalid, "ob_transport_seed: null pointer");
    OB_CUDA(cudaMemsetAsync(field, 0, sizeof(double) * 2 * (size_t)n_vertices, stream));
    OB_CUDA(cudaMemsetAsync(scalars, 0, sizeof(double) * 2 * (size_t)n_vertices, stream));
    OB_CUDA(cudaMemsetAsync(invalid, 0, sizeof(int32_t), stream));
    transport_seed_kernel<<<blocks_for(n_sources), kThreads, 0, stream>>>(sources, vectors, n_sources, n_vertices,
                                                                          field, scalars, invalid);
    OB_CHECK_LAUNCH("transport seed");
    return OB_OK;
}

int ob_transport_tail(const double* field, const double* scalars, int n_vertices, double resolved_fraction,
                      float* transported, uint8_t* resolved, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 1, "ob_transport_tail: bad size");
    OB_REQUIRE(field && scalars && transported && resolved, "ob_transport_tail: null pointer");
    transport_tail_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(field, scalars, n_vertices,
                                                                           resolved_fraction, transported, resolved);
    OB_CHECK_LAUNCH("transport tail");
    return OB_OK;
}

int ob_vertex_unit_gradient(const float* xyz, const int32_t* faces, int n_faces, int n_vertices, const float* normals,
                            const float* areas, const double* values, const int32_t* corner_offsets,
                            const int32_t* corner_slots, float* face_scratch, float* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 1 && n_vertices >= 1, "ob_vertex_unit_gradient: bad size");
    OB_REQUIRE(xyz && faces && normals && areas && values && corner_offsets && corner_slots && face_scratch && out,
               "ob_vertex_unit_gradient: null pointer");
    face_gradient_area_kernel<<<blocks_for(n_faces), kThreads, 0, stream>>>(xyz, faces, n_faces, normals, areas,
                                                                             values, face_scratch);
    OB_CHECK_LAUNCH("face unit gradient");
    gather_corners_vec3_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(face_scratch, corner_offsets,
                                                                                corner_slots, n_vertices, out);
    OB_CHECK_LAUNCH("gather vertex gradient");
    return OB_OK;
}

int ob_log_map_angles(const float* vertex_gradient, const float* basis_x, const float* basis_y,
                      const double* transported, const double* distance, int n_vertices, float* out,
                      ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 1, "ob_log_map_angles: bad size");
    OB_REQUIRE(vertex_gradient && basis_x && basis_y && transported && distance && out,
               "ob_log_map_angles: null pointer");
    log_map_angles_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(vertex_gradient, basis_x, basis_y,
                                                                           transported, distance, n_vertices, out);
    OB_CHECK_LAUNCH("log map angles");
    return OB_OK;
}

int ob_log_map_outward_ball(const float* xyz, const int32_t* faces, const int32_t* ring_offsets,
                            const int32_t* ring_halfedges, const double* tangent_angles,
                            const double* transport_angles, int source, int n_vertices, double* rhs,
                            ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 1 && source >= 0 && source < n_vertices, "ob_log_map_outward_ball: bad source");
    OB_REQUIRE(xyz && faces && ring_offsets && ring_halfedges && tangent_angles && transport_angles && rhs,
               "ob_log_map_outward_ball: null pointer");
    OB_CUDA(cudaMemsetAsync(rhs, 0, sizeof(double) * 4 * (size_t)n_vertices, stream));
    outward_ball_kernel<<<1, 32, 0, stream>>>(xyz, faces, ring_offsets, ring_halfedges, tangent_angles,
                                              transport_angles, source, rhs);
    OB_CHECK_LAUNCH("outward ball");
    return OB_OK;
}

int ob_radial_divergence(const float* xyz, const int32_t* faces, int n_faces, int n_vertices,
                         const double* tangent_angles, const double* transport_angles, const double* fields, int source,
                         const float* cot, const int32_t* corner_offsets, const int32_t* corner_slots,
                         double* corner_scratch, double* divergence, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 1 && n_vertices >= 1 && source >= 0 && source < n_vertices,
               "ob_radial_divergence: bad argument");
    OB_REQUIRE(xyz && faces && tangent_angles && transport_angles && fields && cot && corner_offsets && corner_slots &&
                   corner_scratch && divergence,
               "ob_radial_divergence: null pointer");
    radial_divergence_kernel<<<blocks_for(n_faces), kThreads, 0, stream>>>(xyz, faces, n_faces, tangent_angles,
                                                                            transport_angles, fields, source, cot,
                                                                            corner_scratch);
    OB_CHECK_LAUNCH("radial divergence");
    gather_corners_scalar_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(corner_scratch, corner_offsets,
                                                                                  corner_slots, n_vertices, divergence);
    OB_CHECK_LAUNCH("gather radial divergence");
    return OB_OK;
}

int ob_tangent_to_world(const float* tangent, const float* basis_x, const float* basis_y, int n_vertices, float* out,
                        ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0, "ob_tangent_to_world: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(tangent && basis_x && basis_y && out, "ob_tangent_to_world: null pointer");
    tangent_to_world_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(tangent, basis_x, basis_y, n_vertices, out);
    OB_CHECK_LAUNCH("tangent to world");
    return OB_OK;
}

int ob_log_map_fields(const double* fields, const double* distance, int source, int n_vertices, float* out,
                      ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 1 && source >= 0 && source < n_vertices, "ob_log_map_fields: bad argument");
    OB_REQUIRE(fields && distance && out, "ob_log_map_fields: null pointer");
    log_map_fields_kernel<<<blocks_for(n_vertices), kThreads, 0, stream>>>(fields, distance, source, n_vertices, out);
    OB_CHECK_LAUNCH("log map fields");
    return OB_OK;
}

}  // extern "C"
