// f4: the intrinsic tufted cover of use_robust at method="potpourri3d".
//
// geometry-central's robust heat method (ordito/heat.py:5084 _tufted_intrinsic_delaunay, :3749
// _cover_operators; ordito/kernels/heat.py:710-1204): every face doubled into a front copy and a
// reversed back copy over the same vertices, each edge glued front to front (or front to back
// where its two faces wind it the same way, a rim edge to its own face's back copy, an edge of
// three or more faces along a chain), the float64 lengths mollified and flipped to intrinsic
// Delaunay in rounds of independent sets, and the mass, Laplacian, time step, gradient and
// divergence formed from the flipped lengths alone.
//
// Layout: cover face f < F is mesh face f's front copy (c0, c1, c2), F + f its back copy
// (c0, c2, c1). Slot 3 g + e is cover face g's edge opposite its corner e, running from corner
// e + 1 to corner e + 2; lengths[3 g + e] is its length and twin[3 g + e] the slot across it.
// Mesh halfedge 3 f + k runs corner k to corner k + 1 (its mate code: the other halfedge of a
// two-face edge, -1 on the rim, -2 - lowest on an edge of three or more faces).
//
// Every float64 expression that decides a flip, a length or a divergence term is written with
// explicit round-to-nearest operations (no contracted multiply-adds), so the same steps in any
// IEEE float64 arithmetic give the same bits: the flips are reproducible flip for flip.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>

#include "ob_internal.cuh"
#include "ob_scratch.cuh"

namespace ob {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxEdgeFaces = 64;  // halfedges an edge of three or more faces may carry

__device__ __forceinline__ int he_next(int h) { return h - h % 3 + (h + 1) % 3; }
__device__ __forceinline__ int he_prev(int h) { return h - h % 3 + (h + 2) % 3; }
// The back copy of (c0, c1, c2) is (c0, c2, c1): its slot opposite back_corner(e) is the front
// copy's slot opposite e, run the other way (kernels/heat.py:736).
__device__ __forceinline__ int back_corner(int e) { return e == 0 ? 0 : 3 - e; }

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ int run_end_of(const unsigned long long* __restrict__ keys, int start, int count) {
    const unsigned long long key = keys[start];
    int e = start + 1;
    while (e < count && keys[e] == key) ++e;
    return e;
}

// The mesh halfedge of a pattern run's corner q (the edge opposite corner q % 3 of face q / 3).
__device__ __forceinline__ int halfedge_of_corner(int q) { return 3 * (q / 3) + (q % 3 + 1) % 3; }

// Mate codes (ordito/halfedge.py:609) from the operator pattern: each strict-upper entry's run
// lists the corners opposite its vertex pair, whichever way each face winds the edge.
__global__ void mates_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                             const int* __restrict__ run_start, const unsigned long long* __restrict__ keys,
                             int n_keys, const int* __restrict__ order, int n_vertices, int* __restrict__ mates) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_vertices) return;
    for (int k = offsets[i]; k < offsets[i + 1]; ++k) {
        if (columns[k] <= i) continue;
        const int s = run_start[k], e = run_end_of(keys, s, n_keys);
        if (e - s == 2) {
            const int a = halfedge_of_corner(order[s]), b = halfedge_of_corner(order[s + 1]);
            mates[a] = b;
            mates[b] = a;
        } else if (e - s >= 3) {
            int lowest = INT_MAX;
            for (int p = s; p < e; ++p) lowest = min(lowest, halfedge_of_corner(order[p]));
            for (int p = s; p < e; ++p) mates[halfedge_of_corner(order[p])] = -2 - lowest;
        }
    }
}

// kernels/heat.py:749-798 (tufted_cover): one thread per mesh slot 3 f + e -- its corner in both
// copies, its length from the widened positions, and the twins of its front and back slots for an
// edge of one or two faces.
__global__ void cover_kernel(const float* __restrict__ xyz, const int* __restrict__ faces, int n_faces,
                             const int* __restrict__ mates, int* __restrict__ cover, double* __restrict__ lengths,
                             int* __restrict__ twin, int* __restrict__ nonmanifold) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 3 * n_faces) return;
    const int f = h / 3, e = h % 3;
    const int back = 3 * (n_faces + f) + back_corner(e);
    cover[h] = faces[h];
    cover[back] = faces[h];
    const int tail = faces[he_next(h)], tip = faces[he_prev(h)];
    const double dx = sub((double)xyz[3 * tip], (double)xyz[3 * tail]);
    const double dy = sub((double)xyz[3 * tip + 1], (double)xyz[3 * tail + 1]);
    const double dz = sub((double)xyz[3 * tip + 2], (double)xyz[3 * tail + 2]);
    const double length = __dsqrt_rn(add(add(mul(dx, dx), mul(dy, dy)), mul(dz, dz)));
    lengths[h] = length;
    lengths[back] = length;
    const int mate = mates[he_next(h)];
    if (mate <= -2) {
        *nonmanifold = 1;
        return;
    }
    if (mate < 0) {
        twin[h] = back;
        twin[back] = h;
        return;
    }
    const int front_mate = he_prev(mate);
    const int back_mate = 3 * (n_faces + front_mate / 3) + back_corner(front_mate % 3);
    if (faces[mate] == tail) {
        twin[h] = back_mate;
        twin[back] = front_mate;
    } else {
        twin[h] = front_mate;
        twin[back] = back_mate;
    }
}

__device__ __forceinline__ int cover_copy(const int* __restrict__ faces, int n_faces, int halfedge, bool forward) {
    const int front = he_prev(halfedge);
    return forward ? front : 3 * (n_faces + halfedge / 3) + back_corner(front % 3);
}

// kernels/heat.py:841-873 (glue_nonmanifold_cover_edges): an edge of three or more faces, its
// halfedges in index order from the lowest h0, each one's copy running against h0 glued to its
// predecessor's copy running along h0 (the lowest's predecessor: the highest). One thread per
// such edge (its strict-upper pattern entry); an edge of more than kMaxEdgeFaces halfedges flags
// `too_many` and is left unglued.
__global__ void glue_kernel(const int* __restrict__ offsets, const int* __restrict__ columns,
                            const int* __restrict__ run_start, const unsigned long long* __restrict__ keys,
                            int n_keys, const int* __restrict__ order, int n_vertices,
                            const int* __restrict__ faces, int n_faces, int* __restrict__ twin,
                            int* __restrict__ too_many) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_vertices) return;
    for (int k = offsets[i]; k < offsets[i + 1]; ++k) {
        if (columns[k] <= i) continue;
        const int s = run_start[k], e = run_end_of(keys, s, n_keys);
        const int m = e - s;
        if (m < 3) continue;
        if (m > kMaxEdgeFaces) {
            *too_many = 1;
            continue;
        }
        int hs[kMaxEdgeFaces];
        for (int p = 0; p < m; ++p) {
            const int x = halfedge_of_corner(order[s + p]);
            int q = p;
            while (q > 0 && hs[q - 1] > x) {
                hs[q] = hs[q - 1];
                --q;
            }
            hs[q] = x;
        }
        const int tail = faces[hs[0]];
        for (int p = 0; p < m; ++p) {
            const int x = hs[p], sib = hs[p > 0 ? p - 1 : m - 1];
            const int backward = cover_copy(faces, n_faces, x, faces[x] != tail);
            const int forward = cover_copy(faces, n_faces, sib, faces[sib] == tail);
            twin[backward] = forward;
            twin[forward] = backward;
        }
    }
}

// kernels/heat.py:876-905 (length_sum_and_violation): the sum and count of the front copies'
// lengths and the largest triangle-inequality violation c - a - b, block partials folded in block
// order by the last block, which also forms the mollification's shift (kernels/heat.py:908-921):
// max(0, worst + epsilon * mean).
__global__ void length_sums_kernel(const double* __restrict__ lengths, int n_rows, double epsilon,
                                   double* __restrict__ partials, unsigned int* counter,
                                   double* __restrict__ out) {
    __shared__ double scratch[32];
    __shared__ int last;
    double total = 0.0, count = 0.0, worst = -INFINITY;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += gridDim.x * blockDim.x) {
        const double a = lengths[3 * r], b = lengths[3 * r + 1], c = lengths[3 * r + 2];
        total = add(total, add(add(a, b), c));
        count = add(count, 3.0);
        worst = fmax(worst, fmax(sub(sub(a, b), c), fmax(sub(sub(b, c), a), sub(sub(c, a), b))));
    }
    const double bt = block_sum(total, scratch);
    const double bc = block_sum(count, scratch);
    const double bw = block_max(worst, scratch, -(double)INFINITY);
    if (threadIdx.x == 0) {
        partials[3 * blockIdx.x] = bt;
        partials[3 * blockIdx.x + 1] = bc;
        partials[3 * blockIdx.x + 2] = bw;
    }
    if (!last_block_arrived(counter, &last)) return;
    if (threadIdx.x != 0) return;
    double t = 0.0, c = 0.0, w = -INFINITY;
    for (int b = 0; b < (int)gridDim.x; ++b) {
        t = add(t, __ldcg(&partials[3 * b]));
        c = add(c, __ldcg(&partials[3 * b + 1]));
        w = fmax(w, __ldcg(&partials[3 * b + 2]));
    }
    out[0] = t;
    out[1] = c;
    out[2] = w;
    out[3] = c > 0.0 ? fmax(0.0, add(w, dvd(mul(epsilon, t), c))) : 0.0;
}

__global__ void shift_lengths_kernel(double* __restrict__ lengths, long long n, const double* __restrict__ sums) {
    const double delta = sums[3];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        lengths[i] = add(lengths[i], delta);
}

// heron_area_float64 (kernels/heat.py:924-928).
__device__ __forceinline__ double heron(double a, double b, double c) {
    const double s = dvd(add(add(a, b), c), 2.0);
    return __dsqrt_rn(fmax(0.0, mul(mul(mul(s, sub(s, a)), sub(s, b)), sub(s, c))));
}

// cover_half_cotangent (kernels/heat.py:931-941): (b^2 + c^2 - a^2) / (8 A) at corner e.
__device__ __forceinline__ double half_cot(const double* __restrict__ L, int g, int e, double area) {
    const double a = L[3 * g + e], b = L[3 * g + (e + 1) % 3], c = L[3 * g + (e + 2) % 3];
    return dvd(sub(add(mul(b, b), mul(c, c)), mul(a, a)), mul(8.0, area));
}

__device__ __forceinline__ double slot_half_cot(const double* __restrict__ L, int h) {
    const int g = h / 3;
    return half_cot(L, g, h % 3, heron(L[3 * g], L[3 * g + 1], L[3 * g + 2]));
}

// unfolded_diagonal (kernels/heat.py:952-964): |ad| of triangles abc and dcb unfolded about bc.
__device__ __forceinline__ double unfolded_diagonal(double ab, double bc, double ca, double bd, double dc) {
    const double ax = dvd(sub(add(mul(ab, ab), mul(bc, bc)), mul(ca, ca)), mul(2.0, bc));
    const double ay = __dsqrt_rn(fmax(0.0, sub(mul(ab, ab), mul(ax, ax))));
    const double dx = dvd(sub(add(mul(bd, bd), mul(bc, bc)), mul(dc, dc)), mul(2.0, bc));
    const double dy = -__dsqrt_rn(fmax(0.0, sub(mul(bd, bd), mul(dx, dx))));
    const double x = sub(ax, dx), y = sub(ay, dy);
    return __dsqrt_rn(add(mul(x, x), mul(y, y)));
}

// kernels/heat.py:967-1026 (cover_flip_candidates): an edge failing the Euclidean Delaunay test
// (the two half-cotangents facing it sum below -epsilon), tested once by its lower slot; the
// lowest candidate slot of each face claims it.
__global__ void flip_candidates_kernel(const double* __restrict__ L, const int* __restrict__ twin, int n_slots,
                                       double epsilon, int* __restrict__ flip, double* __restrict__ new_length,
                                       int* __restrict__ claim, int* __restrict__ remap,
                                       int* __restrict__ flipped_face, int* __restrict__ count) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n_slots) return;
    flip[h] = 0;
    remap[h] = -1;
    if (h % 3 == 0) flipped_face[h / 3] = 0;
    if (h == 0) *count = 0;
    const int t = twin[h];
    if (t <= h) return;
    const int f0 = h / 3, f1 = t / 3;
    if (f0 == f1) return;
    const double weight = add(slot_half_cot(L, h), slot_half_cot(L, t));
    if (!(weight < -epsilon)) return;
    const int e0 = h % 3, e1 = t % 3;
    const double d = unfolded_diagonal(L[3 * f0 + (e0 + 2) % 3], L[3 * f0 + e0], L[3 * f0 + (e0 + 1) % 3],
                                       L[3 * f1 + (e1 + 1) % 3], L[3 * f1 + (e1 + 2) % 3]);
    if (!isfinite(d)) return;
    flip[h] = 1;
    new_length[h] = d;
    atomicMin(&claim[f0], h);
    atomicMin(&claim[f1], h);
}

// kernels/heat.py:1043-1103 (cover_flip_commit): a candidate owning both of its faces flips them,
// (a, b, c) and (d, c, b) becoming (a, b, d) and (d, c, a) in place; each slot that moved records
// its old twin and its move, and the new diagonal's two slots are final twins.
__global__ void flip_commit_kernel(const int* __restrict__ flip, const double* __restrict__ new_length,
                                   const int* __restrict__ claim, const int* __restrict__ twin,
                                   int n_slots, int* __restrict__ cover, double* __restrict__ L,
                                   int* __restrict__ pending, int* __restrict__ remap,
                                   int* __restrict__ flipped_face, int* __restrict__ count) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n_slots || flip[h] == 0) return;
    const int t = twin[h];
    const int f0 = h / 3, f1 = t / 3;
    if (claim[f0] != h || claim[f1] != h) return;
    const int e0 = h % 3, e1 = t % 3;
    const int a = cover[h], b = cover[he_next(h)], c = cover[he_prev(h)], d = cover[t];
    const double ca = L[3 * f0 + (e0 + 1) % 3], ab = L[3 * f0 + (e0 + 2) % 3];
    const double bd = L[3 * f1 + (e1 + 1) % 3], dc = L[3 * f1 + (e1 + 2) % 3];
    const double ad = new_length[h];
    const int moves[4][2] = {{he_next(t), 3 * f0}, {he_prev(h), 3 * f0 + 2}, {he_next(h), 3 * f1}, {he_prev(t), 3 * f1 + 2}};
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        pending[moves[m][1]] = twin[moves[m][0]];
        remap[moves[m][0]] = moves[m][1];
    }
    pending[3 * f0 + 1] = -2 - (3 * f1 + 1);
    pending[3 * f1 + 1] = -2 - (3 * f0 + 1);
    cover[3 * f0] = a;
    cover[3 * f0 + 1] = b;
    cover[3 * f0 + 2] = d;
    cover[3 * f1] = d;
    cover[3 * f1 + 1] = c;
    cover[3 * f1 + 2] = a;
    L[3 * f0] = bd;
    L[3 * f0 + 1] = ad;
    L[3 * f0 + 2] = ab;
    L[3 * f1] = ca;
    L[3 * f1 + 1] = ad;
    L[3 * f1 + 2] = dc;
    flipped_face[f0] = 1;
    flipped_face[f1] = 1;
    atomicAdd(count, 1);
}

// kernels/heat.py:1106-1130 (cover_flip_fixup): every slot's twin after the round, into the other
// twin buffer, and the face claims re-armed.
__global__ void flip_fixup_kernel(const int* __restrict__ twin, const int* __restrict__ pending,
                                  const int* __restrict__ remap, const int* __restrict__ flipped_face, int n_slots,
                                  int* __restrict__ twin_out, int* __restrict__ claim) {
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= n_slots) return;
    const int f = h / 3;
    int other = flipped_face[f] ? pending[h] : twin[h];
    if (other <= -2)
        other = -2 - other;
    else if (remap[other] >= 0)
        other = remap[other];
    twin_out[h] = other;
    if (h % 3 == 0) claim[f] = INT_MAX;
}

__global__ void fill_int_kernel(int* __restrict__ out, int n, int value) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = value;
}

// kernels/heat.py:1133-1151 (cover_face_terms): each cover face's three half-cotangents.
__global__ void cover_cot_kernel(const double* __restrict__ L, int n_cover, double* __restrict__ cot) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_cover) return;
    const double area = heron(L[3 * g], L[3 * g + 1], L[3 * g + 2]);
#pragma unroll
    for (int e = 0; e < 3; ++e) cot[3 * g + e] = half_cot(L, g, e, area);
}

// Each vertex's corner areas summed in ascending corner order (the lumped mass's area sums).
__global__ void cover_area_sums_kernel(const double* __restrict__ L, const int* __restrict__ corner_offsets,
                                       const int* __restrict__ corner_slots, int n_vertices,
                                       double* __restrict__ sums) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_vertices) return;
    double s = 0.0;
    for (int p = corner_offsets[v]; p < corner_offsets[v + 1]; ++p) {
        const int g = corner_slots[p] / 3;
        s = add(s, heron(L[3 * g], L[3 * g + 1], L[3 * g + 2]));
    }
    sums[v] = s;
}

// kernels/heat.py:1154-1204 (cover_unit_gradient_divergence) at one corner: the face laid out in
// the plane from its lengths (p0 at the origin, p1 on the x axis), the field's gradient direction
// there normalised as stable_normalize does (divided by its largest component, then by its
// length), and the corner's share t_{e-1} - t_{e+1} of the terms cot_e dot(edge_e, x).
__device__ __forceinline__ double cover_corner_term(const int* __restrict__ cover, const double* __restrict__ L,
                                                    const double* __restrict__ cot, int g, int corner,
                                                    const double* __restrict__ u, int k, int c) {
    const double l0 = L[3 * g], l1 = L[3 * g + 1], l2 = L[3 * g + 2];
    const double x2 = dvd(sub(add(mul(l2, l2), mul(l1, l1)), mul(l0, l0)), mul(2.0, l2));
    const double y2 = __dsqrt_rn(fmax(0.0, sub(mul(l1, l1), mul(x2, x2))));
    const double e0x = sub(x2, l2), e0y = y2;
    const double e1x = -x2, e1y = -y2;
    const double e2x = l2, e2y = 0.0;
    const double u0 = u[(size_t)cover[3 * g] * k + c], u1 = u[(size_t)cover[3 * g + 1] * k + c],
                 u2 = u[(size_t)cover[3 * g + 2] * k + c];
    // perp(e) = (-e.y, e.x)
    const double gx = add(add(mul(-e0y, u0), mul(-e1y, u1)), mul(-e2y, u2));
    const double gy = add(add(mul(e0x, u0), mul(e1x, u1)), mul(e2x, u2));
    const double largest = fmax(fabs(gx), fabs(gy));
    if (!(largest > 0.0)) return 0.0;
    const double wx = dvd(gx, largest), wy = dvd(gy, largest);
    const double norm = __dsqrt_rn(add(mul(wx, wx), mul(wy, wy)));
    const double xx = dvd(wx, norm), xy = dvd(wy, norm);
    const double t0 = mul(cot[3 * g], add(mul(e0x, xx), mul(e0y, xy)));
    const double t1 = mul(cot[3 * g + 1], add(mul(e1x, xx), mul(e1y, xy)));
    const double t2 = mul(cot[3 * g + 2], add(mul(e2x, xx), mul(e2y, xy)));
    return corner == 0 ? sub(t2, t1) : corner == 1 ? sub(t0, t2) : sub(t1, t0);
}

// div(x) at (vertex, column), its corners summed in ascending corner order.
__global__ void cover_divergence_kernel(const int* __restrict__ cover, const double* __restrict__ L,
                                        const double* __restrict__ cot, const int* __restrict__ corner_offsets,
                                        const int* __restrict__ corner_slots, int n_vertices,
                                        const double* __restrict__ u, int k, double* __restrict__ out) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)n_vertices * k) return;
    const int v = (int)(t / k), c = (int)(t % k);
    double s = 0.0;
    for (int p = corner_offsets[v]; p < corner_offsets[v + 1]; ++p) {
        const int q = corner_slots[p];
        s = add(s, cover_corner_term(cover, L, cot, q / 3, q % 3, u, k, c));
    }
    out[t] = s;
}

int blocks_of(long long n) { return (int)std::max(1LL, (n + kThreads - 1) / kThreads); }

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_cover_build(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                   const uint64_t* keys, int n_keys, const int32_t* order, int n_vertices,
                   const float* xyz, const int32_t* faces, int n_faces, double epsilon_mollify,
                   double epsilon_delaunay, int max_rounds, int32_t* cover_faces, double* lengths,
                   int32_t* twin, int32_t* rounds, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_faces >= 0 && n_vertices >= 0 && max_rounds >= 0, "ob_cover_build: bad size");
    if (rounds) *rounds = 0;
    if (n_faces == 0) return OB_OK;
    OB_REQUIRE(offsets && columns && run_start && keys && order && xyz && faces && cover_faces && lengths && twin,
               "ob_cover_build: null pointer");
    OB_REQUIRE(6LL * n_faces < INT_MAX, "ob_cover_build: %d faces exceed int32 slot indexing", n_faces);
    const int n_slots = 6 * n_faces, n_cover = 2 * n_faces;
    const int grid = std::min(blocks_of(n_faces), 4 * sm_count());
    Scratch scratch(stream);
    int* mates = scratch.take<int>(3 * (size_t)n_faces);
    int* flags = scratch.take<int>(3);  // [0] non-manifold, [1] an edge past kMaxEdgeFaces, [2] flips
    int* twin_b = scratch.take<int>(n_slots);
    int* flip = scratch.take<int>(n_slots);
    int* pending = scratch.take<int>(n_slots);
    int* remap = scratch.take<int>(n_slots);
    int* claim = scratch.take<int>(n_cover);
    int* flipped = scratch.take<int>(n_cover);
    double* new_length = scratch.take<double>(n_slots);
    double* partials = scratch.take<double>(3 * (size_t)grid);
    double* sums = scratch.take<double>(4);
    unsigned int* counter = scratch.take<unsigned int>(1);
    if (int st = scratch.commit()) return st;
    OB_CUDA(cudaMemsetAsync(mates, 0xFF, sizeof(int) * 3 * (size_t)n_faces, stream));
    OB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * 3, stream));
    OB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned int), stream));
    mates_kernel<<<blocks_of(n_vertices), kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), n_keys, order, n_vertices, mates);
    OB_CHECK_LAUNCH("cover mates");
    cover_kernel<<<blocks_of(3LL * n_faces), kThreads, 0, stream>>>(xyz, faces, n_faces, mates, cover_faces, lengths,
                                                                     twin, flags);
    OB_CHECK_LAUNCH("cover");
    glue_kernel<<<blocks_of(n_vertices), kThreads, 0, stream>>>(
        offsets, columns, run_start, reinterpret_cast<const unsigned long long*>(keys), n_keys, order, n_vertices,
        faces, n_faces, twin, flags + 1);
    OB_CHECK_LAUNCH("cover glue");
    length_sums_kernel<<<grid, kThreads, 0, stream>>>(lengths, n_faces, epsilon_mollify, partials, counter, sums);
    OB_CHECK_LAUNCH("cover length sums");
    shift_lengths_kernel<<<std::min(blocks_of(n_slots), 4 * sm_count()), kThreads, 0, stream>>>(lengths, n_slots,
                                                                                                 sums);
    OB_CHECK_LAUNCH("cover mollify");
    fill_int_kernel<<<blocks_of(n_cover), kThreads, 0, stream>>>(claim, n_cover, INT_MAX);
    OB_CHECK_LAUNCH("cover claims");
    int host_flags[2] = {0, 0};
    OB_CUDA(cudaMemcpyAsync(host_flags, flags, sizeof(int) * 2, cudaMemcpyDeviceToHost, stream));
    OB_CUDA(cudaStreamSynchronize(stream));
    OB_REQUIRE(!host_flags[1], "ob_cover_build: an edge carries more than %d halfedges", kMaxEdgeFaces);
    // Rounds until one flips nothing: candidates, commit, fixup into the other twin buffer.
    int* current = twin;
    int* other = twin_b;
    int done = 0, count = 0;
    for (int r = 0; r < max_rounds; ++r) {
        flip_candidates_kernel<<<blocks_of(n_slots), kThreads, 0, stream>>>(
            lengths, current, n_slots, epsilon_delaunay, flip, new_length, claim, remap, flipped, flags + 2);
        OB_CHECK_LAUNCH("cover flip candidates");
        flip_commit_kernel<<<blocks_of(n_slots), kThreads, 0, stream>>>(flip, new_length, claim, current, n_slots,
                                                                         cover_faces, lengths, pending, remap,
                                                                         flipped, flags + 2);
        OB_CHECK_LAUNCH("cover flip commit");
        flip_fixup_kernel<<<blocks_of(n_slots), kThreads, 0, stream>>>(current, pending, remap, flipped, n_slots,
                                                                        other, claim);
        OB_CHECK_LAUNCH("cover flip fixup");
        std::swap(current, other);
        ++done;
        OB_CUDA(cudaMemcpyAsync(&count, flags + 2, sizeof(int), cudaMemcpyDeviceToHost, stream));
        OB_CUDA(cudaStreamSynchronize(stream));
        if (count == 0) break;
    }
    if (current != twin)
        OB_CUDA(cudaMemcpyAsync(twin, current, sizeof(int) * (size_t)n_slots, cudaMemcpyDeviceToDevice, stream));
    if (rounds) *rounds = done;
    return OB_OK;
}

int ob_cover_face_terms(const int32_t* cover_faces, const double* lengths, int n_cover, int n_vertices,
                        const int32_t* corner_offsets, const int32_t* corner_slots, double* cot,
                        double* area_sums, double* length_sums, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_cover >= 0 && n_vertices >= 0, "ob_cover_face_terms: bad size");
    OB_REQUIRE(corner_offsets && area_sums && length_sums, "ob_cover_face_terms: null pointer");
    OB_REQUIRE(n_cover == 0 || (cover_faces && lengths && cot && corner_slots), "ob_cover_face_terms: null pointer");
    if (n_cover > 0) {
        cover_cot_kernel<<<blocks_of(n_cover), kThreads, 0, stream>>>(lengths, n_cover, cot);
        OB_CHECK_LAUNCH("cover cot");
    }
    if (n_vertices > 0) {
        cover_area_sums_kernel<<<blocks_of(n_vertices), kThreads, 0, stream>>>(lengths, corner_offsets, corner_slots,
                                                                               n_vertices, area_sums);
        OB_CHECK_LAUNCH("cover area sums");
    }
    // The time step's mean edge: every slot's length, each cover edge counted from both sides.
    const int grid = std::min(blocks_of(std::max(n_cover, 1)), 4 * sm_count());
    Scratch scratch(stream);
    double* partials = scratch.take<double>(3 * (size_t)grid);
    double* sums = scratch.take<double>(4);
    unsigned int* counter = scratch.take<unsigned int>(1);
    if (int st = scratch.commit()) return st;
    OB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned int), stream));
    length_sums_kernel<<<grid, kThreads, 0, stream>>>(lengths, n_cover, 0.0, partials, counter, sums);
    OB_CHECK_LAUNCH("cover edge sums");
    OB_CUDA(cudaMemcpyAsync(length_sums, sums, 2 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    return OB_OK;
}

int ob_cover_divergence(const int32_t* cover_faces, const double* lengths, const double* cot, int n_vertices,
                        const int32_t* corner_offsets, const int32_t* corner_slots, const double* u,
                        int n_columns, double* out, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n_vertices >= 0 && n_columns >= 1, "ob_cover_divergence: bad size");
    if (n_vertices == 0) return OB_OK;
    OB_REQUIRE(cover_faces && lengths && cot && corner_offsets && corner_slots && u && out,
               "ob_cover_divergence: null pointer");
    cover_divergence_kernel<<<blocks_of((long long)n_vertices * n_columns), kThreads, 0, stream>>>(
        cover_faces, lengths, cot, corner_offsets, corner_slots, n_vertices, u, n_columns, out);
    OB_CHECK_LAUNCH("cover divergence");
    return OB_OK;
}

}  // extern "C"
