// Per-face float32 geometry shared by the assembly and divergence kernels.
//
// The arithmetic follows ordito/kernels/predicates.py:106-130 (triangle_area_vector: the cross
// product at the corner opposite the longest edge), :186 (triangle_double_area),
// ordito/kernels/laplacian.py:94-108 (half_cotangents_of) and ordito/kernels/triangles.py:333-359
// (face_normals_and_area), all in float32 with IEEE division and square root.
#pragma once

#include <cuda_runtime.h>

namespace ob {

struct f3 {
    float x, y, z;
};

__device__ __forceinline__ f3 load_f3(const float* __restrict__ p, int i) {
    return f3{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
}
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 neg(f3 a) { return f3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length(f3 a) { return sqrtf(dot(a, a)); }

// Twice the vector area of (a, b, c), formed at the best-conditioned corner.
__device__ __forceinline__ f3 triangle_area_vector(f3 a, f3 b, f3 c) {
    const f3 ab = sub(b, a), bc = sub(c, b), ca = sub(a, c);
    const float l_ab = dot(ab, ab), l_bc = dot(bc, bc), l_ca = dot(ca, ca);
    if (l_bc >= l_ca && l_bc >= l_ab) return cross(ab, neg(ca));
    if (l_ca >= l_ab) return cross(bc, neg(ab));
    return cross(ca, neg(bc));
}

// Half-cotangent of each corner's angle; zeros for a zero-area face.
__device__ __forceinline__ void half_cotangents(f3 v0, f3 v1, f3 v2, float* c) {
    const float dbl = length(triangle_area_vector(v0, v1, v2));
    const float den = 2.0f * dbl;
    if (den <= 0.0f) {
        c[0] = c[1] = c[2] = 0.0f;
        return;
    }
    c[0] = __fdiv_rn(dot(sub(v1, v0), sub(v2, v0)), den);
    c[1] = __fdiv_rn(dot(sub(v2, v1), sub(v0, v1)), den);
    c[2] = __fdiv_rn(dot(sub(v0, v2), sub(v1, v2)), den);
}

// Unit normal (the zero vector for a degenerate face) and area.
__device__ __forceinline__ void normal_and_area(f3 v0, f3 v1, f3 v2, f3* normal, float* area) {
    f3 n = triangle_area_vector(v0, v1, v2);
    const float norm = length(n);
    if (norm > 0.0f) n = f3{__fdiv_rn(n.x, norm), __fdiv_rn(n.y, norm), __fdiv_rn(n.z, norm)};
    *normal = n;
    *area = 0.5f * norm;
}

}  // namespace ob
