/*
 * ordito_b200 -- C ABI of the B200 heat-method geodesic path.
 *
 * Every entry point is extern "C", takes plain device pointers and sizes, returns an int status
 * (OB_OK = 0) and never throws across the boundary. A failed call leaves a one-line message in
 * ob_last_error() (per thread). Device buffers are caller-owned unless a function says otherwise;
 * all work is enqueued on the given stream (NULL = the legacy default stream) and is asynchronous
 * unless a function documents a host read-back.
 *
 * Each declaration names the reference interface it replaces (paths within the ordito project,
 * ordito 0.5.2). A Python binding of this header is ordito_b200/_lib.py (ctypes).
 */
#ifndef ORDITO_B200_H
#define ORDITO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* ob_stream_t; /* a cudaStream_t */

/* Status codes. */
#define OB_OK 0
#define OB_ERR_INVALID 1         /* bad argument (shape, size, null pointer)            */
#define OB_ERR_CUDA 2            /* a CUDA runtime call failed                           */
#define OB_ERR_NOMEM 3           /* device allocation refused                            */
#define OB_ERR_INDEX 4           /* a vertex index out of [0, n_vertices)                */
#define OB_ERR_NOT_CONVERGED 5   /* iteration cap reached outside tolerance              */
#define OB_ERR_NONFINITE 6       /* a non-finite residual stopped the iteration          */
#define OB_ERR_INDEFINITE 7      /* a factorisation met a non-positive pivot             */
#define OB_ERR_TIMEOUT 8         /* a bounded device wait gave up                        */
#define OB_ERR_BUDGET 9          /* over the memory budget                               */

/* Solver status words written by the device loops (never a trap). */
#define OB_STATUS_CONVERGED 0
#define OB_STATUS_CAPPED 1
#define OB_STATUS_NONFINITE 2
#define OB_STATUS_SETTLED 3
#define OB_STATUS_SETTLE_BOUND 4

const char* ob_last_error(void);
int ob_version(void);

/* ---- runtime plumbing (device memory, copies, streams, events) ---------------------------- */
int ob_device_count(int* count);
int ob_set_device(int device);
int ob_get_device(int* device);
/* Stream-ordered pool allocation: usable on `stream` (and after a sync, anywhere); ob_free
 * releases it in `stream` order, so pass the stream of the buffer's last use. */
int ob_malloc(size_t bytes, void** ptr, ob_stream_t stream);
int ob_free(void* ptr, ob_stream_t stream);
int ob_host_alloc(size_t bytes, void** ptr);             /* pinned host memory              */
int ob_host_free(void* ptr);
/* kind: 0 host->device, 1 device->host, 2 device->device, 3 host->host (cudaMemcpyKind order
 * 1, 2, 3, 0); the copy is enqueued on stream and, with sync != 0, waited for. */
int ob_memcpy(void* dst, const void* src, size_t bytes, int kind, ob_stream_t stream, int sync);
int ob_memset(void* dst, int value, size_t bytes, ob_stream_t stream);
int ob_stream_create(ob_stream_t* stream);
int ob_stream_destroy(ob_stream_t stream);
int ob_stream_synchronize(ob_stream_t stream);
int ob_device_synchronize(void);
int ob_event_create(void** event);
int ob_event_destroy(void* event);
int ob_event_record(void* event, ob_stream_t stream);
int ob_event_elapsed_ms(void* start, void* end, float* ms); /* synchronizes on end           */
int ob_event_query(void* event, int* done);               /* done = 1 once the event has passed */
int ob_event_synchronize(void* event);                    /* waits for the event on the host  */
int ob_stream_wait_event(ob_stream_t stream, void* event); /* later work on stream waits for it */
int ob_mem_info(size_t* free_bytes, size_t* total_bytes); /* the device's free / total memory  */
/* The library allocates from the current device's default stream-ordered pool and keeps what it
 * frees there for its next allocations (ob_mem_info counts that memory as free). ob_mem_trim
 * synchronises the device and hands all but keep_bytes of it back to the driver. */
int ob_mem_trim(size_t keep_bytes);
/* Recording a sequence of this library's calls as one CUDA graph: ob_capture_begin(stream)
 * (a created stream), the calls on that stream, ob_capture_end -> a graph replayed by
 * ob_graph_launch on any stream; *kernels = the kernel launches one replay makes (counted by
 * ob_launch_count at each replay). The recorded calls must not allocate persistent buffers
 * (run them once first) and their pointer arguments are fixed in the graph. */
int ob_capture_begin(ob_stream_t stream);
int ob_capture_end(ob_stream_t stream, void** graph, int* kernels);
int ob_graph_launch(void* graph, ob_stream_t stream);
int ob_graph_destroy(void* graph);
/* Number of this library's kernel launches so far in this process (a counter the launches bump). */
int ob_launch_count(uint64_t* count);

/* ---- a1: mesh operator pattern --------------------------------------------------------------
 * Replaces ordito.laplacian.mesh_operator_pattern(faces, n_vertices) for the "cotmatrix"
 * operator (ordito/laplacian.py:1071, _mesh_operator_pattern :1212, kernels store_operator_keys
 * ordito/kernels/laplacian.py:707, csr_from_keys ordito/array.py:1688). Writes count = 6 F + V
 * keys (row * V + col for both directions of each face edge, payload = corner slot 3 f + e; the
 * diagonal of every referenced vertex; the sentinel V * V otherwise), sorts them stably and
 * places the runs: offsets[V + 1], columns[count] (offsets[V] used), run_start[count], and the
 * sorted keys[count] / order[count]. The diagonal slots' payload is -1. */
int ob_pattern_workspace(int n_vertices, int n_faces, size_t* bytes);
int ob_pattern_build(const int32_t* faces, int n_faces, int n_vertices, int32_t* offsets,
                     int32_t* columns, int32_t* run_start, uint64_t* keys, int32_t* order,
                     void* workspace, size_t workspace_bytes, ob_stream_t stream);

/* ---- a2/a3: per-face terms -------------------------------------------------------------------
 * Replaces kernels/heat.py:92 heat_face_terms (and laplacian.cotmatrix_entries,
 * ordito/laplacian.py:189): the float32 half-cotangent table cot[F, 3] (skipped when cot is NULL),
 * unit normals[F, 3], areas[F] and the exact float64 corner sums of the areas area_sums[V]
 * (zeroed here first). xyz is float32[V, 3], faces int32[F, 3]. */
int ob_face_terms(const float* xyz, const int32_t* faces, int n_faces, int n_vertices, float* cot,
                  float* normals, float* areas, double* area_sums, ob_stream_t stream);

/* ---- method="igl" and method="potpourri3d": the operators' variants ---------------------------
 * ob_voronoi_area_sums replaces kernels/heat.py:92 heat_face_terms at voronoi_mass = 1 (with
 * kernels/triangles.py:276 face_voronoi_areas): area_sums[V] (zeroed here) gets each corner's
 * Voronoi share of its face (Meyer et al.'s mixed areas: circumcentric split of a non-obtuse face,
 * half to an obtuse corner and a quarter to the others, an even split of a degenerate face),
 * formed in float64, rounded to float32 and added exactly in float64 -- the lumped mass itself
 * (mass divisor 1 in ob_heat_rows).
 * ob_rim_vertices replaces kernels/heat.py:469 rim_vertices: rim[V] = 1 where a vertex has an edge
 * on a single face (a run of one key in the cotmatrix pattern), *n_rim (device) their count.
 * ob_pinned_rows replaces kernels/heat.py:488 pinned_heat_rows: the heat system with the solution
 * pinned to zero on the rim (rim rows the identity's, rim columns dropped), over the same pattern.
 * ob_off_rim replaces kernels/heat.py:512 off_rim: out = in, zero on the rim.
 * ob_add_to_diagonal replaces the add_to_diagonal kernel of heat.py:4098 (geometry-central's
 * regularized Poisson system -L + 1e-6 I): out = values with shift added to the diagonal. */
int ob_voronoi_area_sums(const float* xyz, const int32_t* faces, int n_faces, int n_vertices,
                         double* area_sums, ob_stream_t stream);
int ob_rim_vertices(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                    const uint64_t* keys, int count, int n_vertices, int32_t* rim, int32_t* n_rim,
                    ob_stream_t stream);
int ob_pinned_rows(const int32_t* offsets, const int32_t* columns, const int32_t* rim, const double* values,
                   int n_vertices, double* out, ob_stream_t stream);
int ob_off_rim(const double* in, const int32_t* rim, int n_vertices, double* out, ob_stream_t stream);
int ob_add_to_diagonal(const int32_t* offsets, const int32_t* columns, const double* values, int n_vertices,
                       double shift, double* out, ob_stream_t stream);
/* ob_mollified_cot replaces ordito.laplacian.mollify_intrinsic (ordito/laplacian.py:779) followed
 * by cotmatrix_entries_intrinsic (:276), the use_robust operators' half-cotangent table: each
 * face's float32 side lengths (lengths[F][3], column e opposite corner e; caller-provided scratch),
 * delta = max(epsilon * mean length - smallest triangle-inequality margin, 0) added to every length
 * (float32; the mean is summed in float64, the reference sums it in float32), and cot[F][3] the
 * float32 half-cotangents by the law of cosines over Kahan's Heron area. *delta_out = delta (one
 * synchronous read-back). */
int ob_mollified_cot(const float* xyz, const int32_t* faces, int n_faces, double epsilon, float* lengths,
                     float* cot, double* delta_out, ob_stream_t stream);

/* ---- a4: edge-length sums for the default time step -----------------------------------------
 * Replaces kernels/heat.py:173 upper_edge_length_sum_and_count (heat.py:2248 _edge_length_sums):
 * out[0] = sum of weight * |v_col - v_row| over the strict upper triangle, out[1] = sum of
 * weights; weight = run length (faces holding the edge) with face_edges != 0, else 1. Summed in a
 * fixed order (bit-reproducible). */
int ob_edge_sums(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                 const uint64_t* keys, int count, int n_vertices, const float* xyz,
                 int face_edges, double* out, ob_stream_t stream);

/* ---- a5: operator rows ------------------------------------------------------------------------
 * Replaces kernels/heat.py:361 heat_system_rows: over the pattern, L (cotangent Laplacian,
 * off-diagonal = run sum of f64(cot) in sorted order, diagonal = -row sum), H = factor L + M and
 * P = -L, with factor = scale (from_edges == 0) or scale * (out[0] / out[1])^2 from ob_edge_sums
 * (from_edges != 0); mass[V] = area_sums / mass_divisor. L/H/P have offsets[V] entries. */
int ob_heat_rows(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                 const uint64_t* keys, int count, const int32_t* order, int n_vertices,
                 const float* cot, double scale, const double* edge_sums, int from_edges,
                 const double* area_sums, double mass_divisor, double* L, double* H, double* P,
                 double* mass, ob_stream_t stream);
/* ob_heat_rows over a float64 half-cotangent table: the intrinsic cover's rows
 * (ordito/heat.py:3786-3813, HEAT_SYSTEM_ROWS[wp.float64]). */
int ob_heat_rows_f64(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                     const uint64_t* keys, int count, const int32_t* order, int n_vertices,
                     const double* cot, double scale, const double* edge_sums, int from_edges,
                     const double* area_sums, double mass_divisor, double* L, double* H, double* P,
                     double* mass, ob_stream_t stream);

/* ---- a6: source indicator -------------------------------------------------------------------
 * Replaces kernels/heat.py:614 seed_source_indicator: u0[V] zeroed then u0[s] = 1 for each source;
 * an index outside [0, V) writes nothing and sets invalid[0] = 1 (invalid is zeroed here). */
int ob_seed(const int32_t* sources, int n_sources, int n_vertices, double* u0, int32_t* invalid,
            ob_stream_t stream);

/* ---- a8: unit gradient and divergence ---------------------------------------------------------
 * Replaces kernels/heat.py:658 unit_gradient_divergence: neg_div[V] (zeroed here) accumulates
 * -div(X) of the per-face normalised gradient of u (float64). With n_columns > 1, u and neg_div
 * hold n_columns fields laid out [V][n_columns] (one vertex's columns contiguous). */
int ob_grad_div(const float* xyz, const int32_t* faces, int n_faces, int n_vertices,
                const float* normals, const float* areas, const double* u, const float* cot,
                int n_columns, double* neg_div, ob_stream_t stream);

/* ---- a13: shift to the sources ------------------------------------------------------------
 * Replaces heat.py:3134 _shift_to_sources (kernels source_and_global_sums :3384 and
 * shift_and_orient :3410): phi -= mean(phi[sources]); with orient != 0 the field is flipped when
 * its mean falls below that offset. With n_columns > 1 phi is [V][n_columns] and column c uses
 * sources[source_offsets[c] .. source_offsets[c + 1]) (a device array; NULL for one column, which
 * then uses the n_sources entries of sources). Every column needs at least one source. The sums
 * are folded in a fixed order. */
int ob_shift(double* phi, int n_vertices, const int32_t* sources, int n_sources,
             const int32_t* source_offsets, int n_columns, int orient, ob_stream_t stream);

/* ob_shift with no device allocation (no counterpart in the reference: this is an entry point for
 * callers that cannot let a library allocate device memory, e.g. a host runtime that owns and
 * accounts all device memory, or a latency-critical loop that may not risk an allocation's
 * driver call). Same arguments and result as ob_shift, at most 64 columns (more are rejected with
 * OB_ERR_INVALID). Its scratch is a static device array of about 129 KiB that every device
 * loading the library holds until exit, shared by every call on that device: calls whose work
 * overlaps on the device race on it and must be ordered by the caller. The first call on each
 * device looks the array's address up, and so does the first call after the device's context
 * changed (a cudaDeviceReset by the host): make those calls before any stream capture. */
int ob_shift_noalloc(double* phi, int n_vertices, const int32_t* sources, int n_sources,
                     const int32_t* source_offsets, int n_columns, int orient, ob_stream_t stream);

/* ---- a7/a9: preconditioned conjugate gradient ---------------------------------------------
 * Replaces ordito/linalg.py:3619 _BatchedCg with the kernels of
 * kernels/algorithms/conjugate_gradient.py (cg_matvec_dots :453, cg_update :797, settle
 * :1509/:1564) and the Jacobi-Chebyshev preconditioner (linalg.py:5135, multigrid.py:988).
 * A solver copies the CSR arrays into its own and owns its work vectors; its iteration's mat-vecs
 * read a sliced-ELL copy it builds from them (slices of 32 rows as wide as their widest row,
 * column-major within a slice, padded with zero entries on the row itself).
 * precond: 0 Jacobi, 1 Jacobi-Chebyshev (degree 12, interval [max(min(80/n, .5), 1-r), 1+r]).
 * narrow != 0 iterates on float32 copies of the values (vectors, dots, scalars stay float64).
 * n_columns right-hand sides are solved together; rhs/x are laid out [n][n_columns]. */
int ob_pcg_create(int n, const int32_t* offsets, const int32_t* columns, const double* values,
                  int n_columns, int precond, int narrow, void** solver, ob_stream_t stream);
int ob_pcg_destroy(void* solver);
/* A solver keeps its own copy of the operator it was created for. ob_pcg_rebind copies another
 * operator of the same shape (n, nnz) into it and redoes the value-dependent setup (inverse
 * diagonal, Chebyshev steps, sliced-ELL copy; reading back the copy's size synchronises the
 * stream, and a copy that must grow drops the recorded loops) -- its recorded loops replay unchanged,
 * which is how an operator rebuilt per call (ordito/linalg.py:1389-1396: "copied into a kept
 * state of that shape, which replays too") avoids a new state and a new recording. */
int ob_pcg_rebind(void* solver, const int32_t* offsets, const int32_t* columns,
                  const double* values, long long nnz, ob_stream_t stream);
/* solve_spd (linalg.py:1356): stops a column at |r| <= tol |b| (2-norm), or at maxiter rounds.
 * Host read-back of iterations[n_columns] and residual[n_columns] (|r| / |b|) when non-NULL. */
int ob_pcg_solve(void* solver, const double* rhs, double* x, double tol, int maxiter,
                 int* iterations, double* relative_residual, ob_stream_t stream);
/* solve_spd_settled (linalg.py:2490): tolerance 0; every check_rounds rounds stop once no entry
 * is newly non-zero and none moved by change_tolerance of itself, or settle_rounds rounds after
 * the non-zero count last changed, or at maxiter. Host read-back of *rounds and *status. */
int ob_pcg_settle(void* solver, const double* rhs, double* x, int check_rounds,
                  double change_tolerance, int settle_rounds, int maxiter, int* rounds,
                  int* status, ob_stream_t stream);
/* Measurement hooks (no counterpart in the reference): the average duration of `reps` standalone
 * launches of the solver's round mat-vec-with-dots kernel on its current vectors (CUDA events on
 * `stream`), and the solver's shape: info[0..5] = n, padded columns, nnz, narrow, blocks, and the
 * sliced-ELL copy's entries (padding included). */
int ob_pcg_time_matvec(void* solver, int reps, float* ms, ob_stream_t stream);
int ob_pcg_info(void* solver, long long* info);
/* backward_error_exceeds (kernels/linalg.py:1167): flag[0] = 1 when some row has
 * |b - A x|_i > tol (|A| |x| + |b|)_i (or is NaN). flag is zeroed here. */
int ob_backward_error(int n, const int32_t* offsets, const int32_t* columns, const double* values,
                      const double* x, const double* rhs, int n_columns, double tol,
                      int32_t* flag, ob_stream_t stream);
/* Element-wise out[i] = in[i] * scale with a type conversion; types 0 = float32, 1 = float64.
 * A utility of the host layer (no counterpart in the reference's path; it keeps every value the
 * host layer returns formed on the device). */
int ob_cast_scale(const void* in, int in_type, void* out, int out_type, long long n, double scale,
                  ob_stream_t stream);
/* Host-layer utilities (no counterpart in the reference's path; they keep every value the host
 * layer returns formed on the device): out = a x + b y elementwise (y may alias out); the
 * transpose of a rows x cols row-major float64 matrix; and the source indicators of n_columns
 * source sets at once -- column c's sources are sources[source_offsets[c] .. [c + 1]) (device
 * array), u0 is [V][n_columns] and zeroed first, an index outside [0, V) sets invalid[0] = 1
 * (replaces kernels/heat.py:614 seed_source_indicator for several columns). */
int ob_axpby(long long n, double a, const double* x, double b, const double* y, double* out,
             ob_stream_t stream);
/* values[i] = max(values[i], floor) over n float32 values: the clamp of
 * ordito.laplacian.cotmatrix_entries(nonnegative_weights=True) (kernels/laplacian.py:146-163,
 * store_half_cotangents), applied to the half-cotangent table. */
int ob_floor_f32(float* values, long long n, float floor, ob_stream_t stream);
/* Measurement hook: the device's float64 FMA throughput (TFLOP/s) from a register-resident FMA
 * loop over every SM (the compute roofline of the float64 dense products). */
int ob_fp64_peak(float* tflops, ob_stream_t stream);
int ob_transpose(int rows, int cols, const double* in, double* out, ob_stream_t stream);
int ob_seed_columns(const int32_t* sources, const int32_t* source_offsets, int n_columns,
                    int n_vertices, double* u0, int32_t* invalid, ob_stream_t stream);
/* Axis-aligned bounds of float32 points xyz[n, 3]: out[6] = (min xyz, max xyz), as float64 of the
 * float32 extremes. Replaces the mesh bounds the time-step floor reads (ordito/mesh.py:1045,
 * heat.py:5228 _diffusion_floor). */
int ob_bounds(const float* xyz, int n, double* out, ob_stream_t stream);
/* y = A x (float64), n_columns columns [n][n_columns]. */
int ob_spmv(int n, const int32_t* offsets, const int32_t* columns, const double* values,
            const double* x, double* y, int n_columns, ob_stream_t stream);

/* ---- a11: sparse Cholesky ----------------------------------------------------------------
 * Replaces ordito.cholesky (SparseCholesky :121, sparse_cholesky :538, _analyse :881, _factor
 * :1399, _Solve :1606) behind linalg.OperatorFactorization (ordito/linalg.py:2191).
 * ob_chol_analyse: nested-dissection ordering of the pattern (geometric from xyz[n, 3] when not
 * NULL; dissection leaves of at most leaf_size vertices, <= 0 for the default) and the supernodal
 * structure; host work, reads the pattern back. info[0..4] = n,
 * supernodes, tree levels, factor entries, widest front.
 * ob_chol_factor: numeric factorisation of sign * values over the analysed pattern (sign = -1 when
 * negated != 0: a negative (semi-)definite operator such as a cotangent Laplacian; the solves
 * still answer A x = rhs), on the device (multifrontal, level by level, float64 tensor-core
 * products; ordito/cholesky.py:1399 _factor). singular: 0 pins nothing, 1 pins the last vertex of
 * every connected component, 2 pins it on the components whose rows all sum to zero (|row sum| <=
 * 1e-10 |diagonal|, ordito/cholesky.py:76) -- a singular component is then solved up to a
 * constant. A row with no (or a zero) diagonal is always pinned. OB_ERR_INDEFINITE on a pivot
 * that is not positive (one read-back at the end; the call returns when the factor is ready).
 * ob_chol_solve: x = A^-1 rhs for n_columns interleaved columns ([n][n_columns]), then `refine`
 * float64 refinement steps x += A^-1 (rhs - A x) with the operator's CSR arrays (may be NULL when
 * refine == 0); level-scheduled batched dense products on the device, recorded once per
 * (n_columns, refine) as a CUDA graph and replayed, no host read-back. rhs == NULL solves the
 * factor's own right-hand-side buffer and x == NULL leaves the result in its own solution buffer
 * (ob_chol_buffers returns both, sized for n_columns), so a pipeline can chain solves with no
 * copies. ob_chol_time_solve: average duration of `reps` forward+backward triangular passes
 * (CUDA events; a measurement hook). ob_chol_info: info[0..3] = n, stored values, tree levels,
 * product launches per pass. */
int ob_chol_analyse(int n, const int32_t* offsets, const int32_t* columns, const float* xyz,
                    int leaf_size, void** analysis, ob_stream_t stream);
/* ob_chol_analyse_blocked: the analysis of an operator whose rows come in groups of `block`
 * consecutive rows, one group a mesh vertex (xyz holds n / block points) -- the vector heat
 * system's two tangent components a vertex. The dissection runs over the vertices and each
 * vertex's rows stay consecutive in the ordering. ob_chol_analyse is block 1. */
int ob_chol_analyse_blocked(int n, int block, const int32_t* offsets, const int32_t* columns, const float* xyz,
                            int leaf_size, void** analysis, ob_stream_t stream);
int ob_chol_analysis_info(void* analysis, long long* info);
/* The same analysis from host arrays (no device), and the supernodes of an analysis as
 * out[4 s .. 4 s + 3] = (tree level, own columns, off-diagonal rows, parent or -1), postorder.
 * Inspection hooks (no counterpart in the reference). */
int ob_chol_host_analyse(int n, const int32_t* offsets, const int32_t* columns, const float* xyz,
                         int leaf_size, void** analysis);
int ob_chol_analysis_nodes(void* analysis, int32_t* out);
int ob_chol_analysis_destroy(void* analysis);
int ob_chol_factor(void* analysis, const double* values, int singular, int negated, void** factor,
                   ob_stream_t stream);
int ob_chol_nbytes(void* factor, size_t* bytes);
/* The factor's stored values (every supernode's [L11^-1; G] block, padded rows included) copied
 * into out (a device buffer of capacity doubles; NULL only asks *count). An inspection hook (no
 * counterpart in the reference). */
int ob_chol_values(void* factor, double* out, long long capacity, long long* count, ob_stream_t stream);
/* Host check of the same analysis, factorisation and solve algorithm on host arrays (no device;
 * a test hook, no counterpart in the reference): x = A^-1 rhs for one column; info[0..3] as
 * ob_chol_analysis_info's first four (may be NULL). */
int ob_chol_host_solve(int n, const int32_t* offsets, const int32_t* columns,
                       const double* values, const float* xyz, int leaf_size, int singular,
                       const double* rhs, double* x, long long* info);
int ob_chol_destroy(void* factor);
int ob_chol_solve(void* factor, const double* rhs, double* x, int n_columns, int refine,
                  const int32_t* offsets, const int32_t* columns, const double* values,
                  ob_stream_t stream);
int ob_chol_buffers(void* factor, int n_columns, double** rhs, double** solution,
                    ob_stream_t stream);
/* The factor's internal buffers in its own numbering, for pipelines that stay in it: rhs (B) and
 * solution (X) hold row i of the factor's ordering at i * stride (stride = n_columns rounded up
 * to even; a pad column must be zero), iperm maps a vertex to its row, pinned marks the rows
 * whose right-hand side must be zero. ob_chol_solve_in_place: X = A^-1 B in that numbering (no
 * permutation, no refinement), recorded once per n_columns as a CUDA graph. B is consumed. The
 * solution pointer depends on the stride: use the pointers of the n_columns the solve is given. */
int ob_chol_work(void* factor, int n_columns, double** rhs, double** solution, int* stride,
                 const int32_t** iperm, const char** pinned, ob_stream_t stream);
int ob_chol_solve_in_place(void* factor, int n_columns, ob_stream_t stream);

/* ---- the served batch's per-query kernels (ordito_b200/csrc/ob_served.cu) ------------------
 * ob_corner_index: each vertex's corner slots (3 f + e) in ascending order -- a stable sort of
 * the face buffer by vertex (ordito/heat.py:3198 _corner_order) -- as corner_offsets[V + 1] and
 * corner_slots[3 F]; workspace from ob_corner_index_workspace.
 * ob_grad_div_gather: kernels/heat.py:658 unit_gradient_divergence gathered per vertex instead of
 * scattered per face: out[row(v) * out_stride + c] = -div of column c's unit gradient at v,
 * summed over v's corners in ascending slot order (no atomics; bit-reproducible), where
 * row(v) = out_iperm[v] (or v when NULL) and u is read at u_iperm rows with stride u_stride;
 * rows marked in out_pinned (in out's numbering, may be NULL) are written as 0, and so are the
 * pad columns n_columns .. out_stride - 1.
 * ob_seed_permuted: the source indicators of n_columns source sets written into a factor's
 * right-hand side in its numbering (zeroed first; pinned rows stay 0).
 * ob_shift_permuted: heat.py:3134 _shift_to_sources for n_columns columns of phi held in a
 * factor's numbering (stride, iperm), written out transposed as out[c * V + v]. */
/* ob_renumber: out[i] = map[indices[i]] for count indices (no reference counterpart: the served
 * pass renumbers the face buffer into the factors' ordering once per mesh, so its divergence
 * reads and writes factor rows with no inverse permutation per corner). */
int ob_renumber(const int32_t* indices, long long count, const int32_t* map, int32_t* out,
                ob_stream_t stream);
int ob_corner_index_workspace(int n_vertices, int n_faces, size_t* bytes);
int ob_corner_index(const int32_t* faces, int n_faces, int n_vertices, int32_t* corner_offsets,
                    int32_t* corner_slots, void* workspace, size_t workspace_bytes,
                    ob_stream_t stream);
int ob_grad_div_gather(const float* xyz, const int32_t* faces, const float* normals,
                       const float* areas, const float* cot, const int32_t* corner_offsets,
                       const int32_t* corner_slots, int n_vertices, int n_columns, const double* u,
                       int u_stride, const int32_t* u_iperm, double* out, int out_stride,
                       const int32_t* out_iperm, const char* out_pinned, ob_stream_t stream);
/* ob_face_gradient_terms: once per mesh, the divergence's u-independent per-face terms,
 * terms[F][18] float64: the gradient bases n x e_k (e_0 = v2 - v1, e_1 = v0 - v2, e_2 = v1 - v0;
 * zero for a face of no area) and per corner e the cotangent-weighted edge sum W_e, with
 * d_e = W_e . X (kernels/heat.py:626-687 forms the same d_e as two dot products).
 * ob_grad_div_terms: ob_grad_div_gather's result (the same layouts, permutations and pinned rows)
 * from those terms: per corner g = sum_k u_k (n x e_k), rescaled exactly by a power of two to
 * s = g 2^-e (e the exponent of its largest component), d_e = (W_e . s) / |s|. */
int ob_face_gradient_terms(const float* xyz, const int32_t* faces, int n_faces, const float* normals,
                           const float* areas, const float* cot, double* terms, ob_stream_t stream);
int ob_grad_div_terms(const double* terms, const int32_t* faces, const int32_t* corner_offsets,
                      const int32_t* corner_slots, int n_vertices, int n_columns, const double* u,
                      int u_stride, const int32_t* u_iperm, double* out, int out_stride,
                      const int32_t* out_iperm, const char* out_pinned, ob_stream_t stream);
/* ob_corner_records / ob_grad_div_records: ob_grad_div_terms over corner records (no reference
 * counterpart: a layout of the same arithmetic). Set-up, once per face buffer and corner index:
 * records[3 F][12] float64, corner p's twelve terms (its face's gradient bases a, b, w and its
 * W_e) for corner_slots[p], and ids[3 F][4] int32, that face's three vertices (and a zero), both
 * 16-byte aligned. ob_grad_div_records then takes ob_grad_div_terms' arguments with the records,
 * ids and corner offsets in place of the terms, faces and corner index, and returns its bits. */
int ob_corner_records(const double* terms, const int32_t* faces, const int32_t* corner_slots, int n_faces,
                      double* records, int32_t* ids, ob_stream_t stream);
int ob_grad_div_records(const double* records, const int32_t* ids, const int32_t* corner_offsets, int n_vertices,
                        int n_columns, const double* u, int u_stride, const int32_t* u_iperm, double* out,
                        int out_stride, const int32_t* out_iperm, const char* out_pinned, ob_stream_t stream);
/* ob_divergence_tiles / ob_grad_div_tiled: ob_grad_div_terms face by face over tiles of 32
 * consecutive vertices (no reference counterpart: a layout of the same arithmetic). Set-up, once
 * per face buffer and corner index: tile_faces[3 F] (each tile's distinct faces, stored over the
 * start of its corner range), tile_counts[ceil(V / 32)] and corner_codes[3 F]. ob_grad_div_tiled
 * then forms each distinct face's unit gradient once per column and tile (kernels/heat.py:626-687)
 * and sums each vertex's corners in ascending slot order: ob_grad_div_terms' arguments and
 * result (to rounding: the corner contributions are rounded before they are added), no atomics,
 * the same bits on every run. */
int ob_divergence_tiles(const int32_t* corner_offsets, const int32_t* corner_slots, int n_vertices,
                        int32_t* tile_faces, int32_t* tile_counts, int32_t* corner_codes, ob_stream_t stream);
int ob_grad_div_tiled(const double* terms, const int32_t* faces, const int32_t* corner_offsets,
                      const int32_t* corner_slots, const int32_t* tile_faces, const int32_t* tile_counts,
                      const int32_t* corner_codes, int n_vertices, int n_columns, const double* u, int u_stride,
                      const int32_t* u_iperm, double* out, int out_stride, const int32_t* out_iperm,
                      const char* out_pinned, ob_stream_t stream);
int ob_seed_permuted(const int32_t* sources, const int32_t* source_offsets, int n_columns,
                     int n_vertices, const int32_t* iperm, const char* pinned, int stride,
                     double* rhs, ob_stream_t stream);
int ob_shift_permuted(const double* phi, int n_vertices, int stride, const int32_t* iperm,
                      const int32_t* sources, const int32_t* source_offsets, int n_columns,
                      int orient, double* out, ob_stream_t stream);
int ob_chol_time_solve(void* factor, int n_columns, int reps, float* ms, ob_stream_t stream);
/* ob_chol_tile (a tuning hook; no counterpart in the reference): rebuild the passes' tile lists
 * with another split of long inner dimensions -- chunk: the inner range of a split tile (a
 * multiple of 8 from 16 to 4096, or 0: never split; other values are OB_ERR_INVALID), applied at levels with fewer tiles than `waves` waves of the resident
 * grid (0 to 64). Waits for the device, drops the factor's recorded solves and moves every work
 * set's generation (recordings over ob_chol_work buffers must be made again). The defaults after
 * ob_chol_factor are chunk 64, waves 2. */
int ob_chol_tile(void* factor, int chunk, int waves, ob_stream_t stream);
/* ob_chol_tile_columns (a tuning hook; no counterpart in the reference): the column width of the
 * 64-row tensor-core tiles per tree level -- levels with fewer tiles than narrow_waves waves of
 * the resident grid (0 to 64; 0: none) take 32-column tiles (twice the CTAs, each half the
 * columns) instead of 64; the default after ob_chol_factor is 64 (every level). Batches of 1-8
 * columns always take the register kernel, batches of 9-16 columns 16-column tiles. Waits for the device, drops the recorded solves and
 * moves the work generations as ob_chol_tile does. */
int ob_chol_tile_columns(void* factor, int narrow_waves, ob_stream_t stream);
int ob_chol_info(void* factor, long long* info);
/* Deterministic passes (ordito.config.set_deterministic, ordito/config.py:125, for the factored
 * solves): on != 0 rebuilds the passes with no split tiles and with each supernode's forward
 * update written to its own rows, then added into its target rows by one gather launch a tree
 * level in supernode order -- no atomics in a pass, so every solve repeats bit for bit (slower:
 * the long inner dimensions of the upper levels are no longer split). Waits for the device, drops
 * the recorded solves, moves every work set's generation and reallocates the work buffers made
 * so far (deterministic ones hold the update rows too). */
int ob_chol_set_deterministic(void* factor, int on, ob_stream_t stream);
/* The work buffers' generation: it changes whenever ob_chol_work's pointers do (a wider k than
 * any before reallocates them), so a graph recorded over them must be recorded again. */
int ob_chol_work_generation(void* factor, long long* generation);
/* A factor holds six independent sets of work buffers (set 0 is the one every call above uses):
 * passes on different sets share only the read-only factor, so they may run concurrently on two
 * streams -- two batches of one mesh in flight at once (each set on one stream at a time). */
int ob_chol_work_set(void* factor, int set, int n_columns, double** rhs, double** solution,
                     int* stride, const int32_t** iperm, const char** pinned, ob_stream_t stream);
int ob_chol_solve_in_place_set(void* factor, int set, int n_columns, ob_stream_t stream);
/* ob_chol_solve_in_place_sources: ob_chol_solve_in_place_set for a B that holds a batch of source
 * indicators (as ob_seed_permuted writes them for sources / source_offsets, n_columns sets, vertex
 * indices): the forward pass runs only the supernodes a source reaches -- its own and their
 * ancestors -- since every other supernode's input block is zero (their Y rows are written as
 * zero). On a factor analysed without the deterministic flag the backward pass of such a supernode
 * starts past its own zero Y block (only the G^T X[off] part of X = [L11^-1; G]^T [Y; X[off]]
 * runs). Marks on the device (no host read), so it can be recorded. */
int ob_chol_solve_in_place_sources(void* factor, int set, int n_columns, const int32_t* sources,
                                   const int32_t* source_offsets, ob_stream_t stream);
int ob_chol_work_generation_set(void* factor, int set, long long* generation);

/* ---- Smoothed-aggregation multigrid and the mixed-precision solve --------------------------
 *
 * ob_amg_setup replaces ordito.linalg.multigrid_preconditioner(matrix, n_columns, seed=seed)
 * (ordito/linalg.py:5020) and the hierarchy build behind it (_multigrid_hierarchy, :6412): a
 * smoothed-aggregation hierarchy of the n x n symmetric positive (semi-)definite CSR operator
 * (device arrays; float64 values), built once on the host and held on the device in float32.
 * The handle borrows offsets/columns/values (the solve reads them for its float64 residual):
 * they must outlive it. A hierarchy that cannot coarsen (ordito/linalg.py:5118) leaves a Jacobi
 * preconditioner in its place (ob_amg_info: info[0] = 0).
 *
 * ob_amg_info: info[0..3] = levels (0 = Jacobi), coarsest rows, coarsest active rows, stored
 * entries over all levels. ob_amg_levels: rows and stored entries per level (up to capacity).
 *
 * ob_amg_apply: x = M b, one V-cycle on k columns, the ``matvec(x, y, z, 1, 0)`` of the
 * reference's returned operator (ordito/linalg.py:5123). Multi-column arrays are [n][ld] rows
 * (entry (row, c) at row * ld + c, ld >= k), as everywhere in this library.
 *
 * ob_amg_solve replaces ordito.linalg.solve_spd(matrix, rhs, solution, tol=..., preconditioner=
 * multigrid_preconditioner(matrix)) (ordito/linalg.py:1356) for k columns: x is the initial
 * guess and is overwritten. Float64 iterative refinement around a float32 CG preconditioned by
 * the float32 V-cycle: each outer round forms r = b - A x in float64, solves A d = r / |r| in
 * float32 to a relative residual of inner_tol (at most max_inner iterations), and adds |r| d to
 * x in float64; it stops per column at |b - A x|_2 <= tol |b|_2 or after max_outer rounds.
 * Per column: iterations (inner CG iterations, all rounds), residuals (final |r|_2 / |b|_2),
 * statuses (OB_STATUS_CONVERGED, _CAPPED or _NONFINITE). Any pointer among the three may be NULL.
 *
 * ob_amg_host_setup builds the same hierarchy from host arrays and reports its level shape
 * (no device needed).
 *
 * ob_amg_time_kernels (measurement; no counterpart in the reference): the finest level's V-cycle
 * kernels on k float32 columns (zeroed inputs), each launched reps times after one warm-up and
 * timed with CUDA events on stream: ms[0..4] = average milliseconds of a damped-Jacobi sweep,
 * the residual, the restriction product, the prolongation product (accumulating) and one whole
 * V-cycle; bytes[0..3] = each kernel's algorithmic bytes (every stored entry, offset and vector
 * row read or written once; bytes[4] = 0). Needs a hierarchy of two levels or more. */
int ob_amg_setup(int n, const int32_t* offsets, const int32_t* columns, const double* values,
                 unsigned seed, void** amg, ob_stream_t stream);
/* Where ob_amg_setup builds a hierarchy's levels of 32 768 rows or more (process-wide; no
 * counterpart in the reference, which builds on the device): on_device != 0 (the default) on the
 * device -- strength, the MIS-2 rounds, the label spread, the power steps, the smoothed
 * prolongator, its transpose and the Galerkin products assembled by sort-and-segment, each with
 * the host build's arithmetic in its order -- then the smaller levels and the coarse
 * pseudo-inverse on the host; 0 the whole build on host threads. */
int ob_amg_build_mode(int on_device);
int ob_amg_destroy(void* amg);
int ob_amg_info(void* amg, long long* info);
int ob_amg_levels(void* amg, long long* rows, long long* nnz, int capacity);
int ob_amg_apply(void* amg, const double* b, double* x, int k, int ld, ob_stream_t stream);
int ob_amg_solve(void* amg, const double* b, double* x, int k, int ld, double tol, int max_outer,
                 int max_inner, double inner_tol, int* iterations, double* residuals,
                 int* statuses, ob_stream_t stream);
int ob_amg_host_setup(int n, const int32_t* offsets, const int32_t* columns, const double* values,
                      unsigned seed, long long* rows, long long* nnz, int capacity, int* levels);
int ob_amg_time_kernels(void* amg, int k, int reps, float* ms, long long* bytes, ob_stream_t stream);

/* ---- Packed meshes: many meshes solved as one block-diagonal system -------------------------
 * The batched form of ordito.heat.heat_geodesic over many meshes at once: the meshes' vertices
 * and faces concatenated (each face offset by its mesh's first vertex), so the pattern, the face
 * terms, the factorisation and the passes run once over the union; column c carries every mesh's
 * c-th single-source query.
 * ob_edge_sums_segments: ob_edge_sums per segment of rows (a mesh: rows [segments[s],
 * segments[s + 1])), out[2 s], out[2 s + 1], added in a fixed order.
 * ob_heat_rows_packed: ob_heat_rows with each row's own factor (its mesh's -t): L, H = factor L
 * + M, P = -L and the mass, the same arithmetic per row.
 * ob_shift_packed: ob_shift_permuted per (mesh, column): sources[m * n_columns + c] is the local
 * source vertex of mesh m's query in column c (-1: none, its distances are written 0); each
 * mesh's field is shifted by its source's value and oriented by its own mean
 * (kernels/heat.py:3384-3424); out is (n_columns, V); sums is 2 * n_meshes * n_columns doubles
 * of scratch. A mesh's sum is taken over chunks of 2048 of its rows (each chunk's sums apart,
 * then added in chunk order: the same order for a given packing), so large meshes do not hold
 * the launch; the call allocates its chunk table in stream order. */
int ob_edge_sums_segments(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                          const uint64_t* keys, int count, const float* xyz, int face_edges,
                          const int32_t* segments, int n_segments, double* out, ob_stream_t stream);
int ob_heat_rows_packed(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                        const uint64_t* keys, int count, const int32_t* order, int n_vertices,
                        const float* cot, const double* row_factor, const double* area_sums,
                        double mass_divisor, double* L, double* H, double* P, double* mass,
                        ob_stream_t stream);
int ob_shift_packed(const double* phi, int n_vertices, int stride, const int32_t* iperm,
                    const int32_t* vertex_offsets, int n_meshes, const int32_t* sources,
                    int n_columns, double* sums, double* out, ob_stream_t stream);

/* ---- f3: scalar extension -------------------------------------------------------------------
 * ob_extend_seed replaces kernels/heat.py:3858 seed_source_scalars (ordito/heat.py:2426
 * _extend_scalar): rhs[V][2] (zeroed here) gets column 0 = the indicator of the sources, column 1
 * = the values they carry (a repeated source adds up), range[0..1] = the values' min and max and
 * range[2] = 0; an index outside [0, V) sets invalid[0] (zeroed here).
 * ob_extend_ratio replaces kernels/heat.py:3933 extend_from_ratio: extended[i] = diffused[i][1] /
 * diffused[i][0] (0 where the diffused indicator is exactly 0), and range[2] = the largest excess
 * of the extension over [range[0], range[1]] at vertices the indicator reaches. */
int ob_extend_seed(const int32_t* sources, const double* values, int n_sources, int n_vertices, double* rhs,
                   double* range, int32_t* invalid, ob_stream_t stream);
int ob_extend_ratio(const double* diffused, int n_vertices, double* range, double* extended, ob_stream_t stream);

/* ---- f3: the vector heat method (transport_tangent_vectors, log_map) ----------------------
 * Halfedge h = 3 f + k runs faces[3 f + k] -> faces[3 f + (k + 1) % 3].
 * ob_halfedge_twins replaces ordito/halfedge.py:59 halfedge_twins, from the operator pattern
 * (ob_pattern_build's offsets, columns, run_start, sorted keys and order): twins[3F] = the
 * opposite halfedge, -1 on the boundary; defects[0] = edges carried by three or more halfedges,
 * defects[1] = edges whose two halfedges run the same way (a caller rejects the mesh when either
 * is non-zero, as the reference raises ValueError).
 * ob_vertex_one_rings replaces ordito/halfedge.py:284 vertex_one_rings: ring_halfedges[3F] laid
 * out by the corner index (ob_corner_index: each vertex's degree and ascending corners), each
 * vertex's outgoing halfedges counter-clockwise from its outgoing boundary halfedge on a rim, else
 * from its lowest-indexed one; is_boundary[V]; defects[0] = pinched vertices (their remaining
 * slots -1).
 * ob_halfedge_tangent_angles replaces ordito/tangent_space.py:254 halfedge_tangent_angles: each
 * halfedge's float64 polar angle in its origin's frame (corner_angles[3F] is scratch; a caller's
 * float32 face_angles[F][3], or NULL to form them in float64 from the positions).
 * ob_vertex_tangent_frames replaces ordito/tangent_space.py:38 vertex_tangent_frames: basis_x,
 * basis_y float32 [V][3] around given_normals[V][3], or (NULL) around the angle-weighted normals
 * gathered over the rings and written to normals[V][3].
 * ob_tangent_to_world replaces heat.py tangent_to_world (kernels/heat.py:583): out[V][3] =
 * tangent[v][0] basis_x[v] + tangent[v][1] basis_y[v].
 * ob_halfedge_transport replaces ordito/tangent_space.py:363 halfedge_transport_angles and
 * heat.py:1958 _transport_rotations: rho[3F] and rotations[3F][2] = (cos, sin); either may be
 * NULL.
 * ob_polar_unit: rotations[n][2] = (cos, sin) of caller-supplied transport angles (heat.py:1958).
 * ob_half_cot_f64: the float64 half-cotangent table [F][3] (kernels/laplacian.py:130).
 * ob_block_pattern: the pattern expanded to 2 V rows (vertex v's rows 2v and 2v + 1, entry k's
 * 2 x 2 block at columns 2c, 2c + 1): block_offsets[2V + 1], block_columns[4 nnz].
 * ob_vector_heat_rows replaces kernels/heat.py:524 vector_heat_system_rows: the values[4 nnz] of
 * M + factor L_connection over the expanded pattern, factor = scale or, with from_edges,
 * scale * (edge_sums[0] / edge_sums[1])^2; mass[V] is the scalar bundle's lumped mass.
 * ob_transport_seed replaces kernels/heat.py:3881 seed_transport_sources: field[2V] (the vectors,
 * interleaved) and scalars[V][2] (indicator, magnitude), both zeroed here; invalid[0] set by an
 * out-of-range source.
 * ob_transport_tail replaces kernels/heat.py:3975 transported_and_resolved: transported[V][2]
 * float32 and resolved[V] (uint8).
 * ob_vertex_unit_gradient replaces kernels/heat.py:3999 scatter_unit_gradient_to_vertices with
 * the corner sum in ascending corner order: out[V][3] float32 (face_scratch [F][3] float32).
 * ob_log_map_angles replaces kernels/heat.py:4030 log_map_from_angles: out[V][2] float32.
 * ob_log_map_outward_ball replaces kernels/heat.py:4088 seed_log_map_outward_ball: rhs[2V][2]
 * (zeroed here), column 0 the outward ball, column 1 the source's reference direction.
 * ob_radial_divergence replaces kernels/heat.py:4193 radial_field_divergence over fields[2V][2]
 * (corner_scratch [3F] float64; summed per vertex in ascending corner order).
 * ob_log_map_fields replaces kernels/heat.py:4228 log_map_from_vector_fields: out[V][2] float32. */
int ob_halfedge_twins(const int32_t* offsets, const int32_t* columns, const int32_t* run_start, const uint64_t* keys,
                      int n_keys, const int32_t* order, const int32_t* faces, int n_faces, int n_vertices,
                      int32_t* twins, int32_t* defects, ob_stream_t stream);
int ob_vertex_one_rings(const int32_t* corner_offsets, const int32_t* corner_slots, const int32_t* twins,
                        int n_vertices, int32_t* ring_halfedges, uint8_t* is_boundary, int32_t* defects,
                        ob_stream_t stream);
int ob_halfedge_tangent_angles(const float* xyz, const int32_t* faces, int n_faces, int n_vertices,
                               const int32_t* ring_offsets, const int32_t* ring_halfedges, const uint8_t* is_boundary,
                               const float* face_angles, double* corner_angles, double* angles, ob_stream_t stream);
int ob_vertex_tangent_frames(const float* xyz, const int32_t* faces, int n_faces, int n_vertices,
                             const int32_t* ring_offsets, const int32_t* ring_halfedges, const uint8_t* is_boundary,
                             const float* given_normals, float* basis_x, float* basis_y, float* normals,
                             ob_stream_t stream);
int ob_tangent_to_world(const float* tangent, const float* basis_x, const float* basis_y, int n_vertices, float* out,
                        ob_stream_t stream);
int ob_halfedge_transport(const int32_t* twins, const double* tangent_angles, int n_halfedges, double* rho,
                          double* rotations, ob_stream_t stream);
int ob_polar_unit(const double* angles, int n, double* rotations, ob_stream_t stream);
int ob_half_cot_f64(const float* xyz, const int32_t* faces, int n_faces, double* cot, ob_stream_t stream);
int ob_block_pattern(const int32_t* offsets, const int32_t* columns, int n_vertices, int32_t* block_offsets,
                     int32_t* block_columns, ob_stream_t stream);
int ob_vector_heat_rows(const int32_t* offsets, const int32_t* columns, const int32_t* run_start, const uint64_t* keys,
                        int n_keys, const int32_t* order, int n_vertices, const int32_t* faces, const double* cot,
                        const double* rotations, const double* mass, double scale, const double* edge_sums,
                        int from_edges, double* values, ob_stream_t stream);
int ob_transport_seed(const int32_t* sources, const float* vectors, int n_sources, int n_vertices, double* field,
                      double* scalars, int32_t* invalid, ob_stream_t stream);
int ob_transport_tail(const double* field, const double* scalars, int n_vertices, double resolved_fraction,
                      float* transported, uint8_t* resolved, ob_stream_t stream);
int ob_vertex_unit_gradient(const float* xyz, const int32_t* faces, int n_faces, int n_vertices, const float* normals,
                            const float* areas, const double* values, const int32_t* corner_offsets,
                            const int32_t* corner_slots, float* face_scratch, float* out, ob_stream_t stream);
int ob_log_map_angles(const float* vertex_gradient, const float* basis_x, const float* basis_y,
                      const double* transported, const double* distance, int n_vertices, float* out,
                      ob_stream_t stream);
int ob_log_map_outward_ball(const float* xyz, const int32_t* faces, const int32_t* ring_offsets,
                            const int32_t* ring_halfedges, const double* tangent_angles,
                            const double* transport_angles, int source, int n_vertices, double* rhs,
                            ob_stream_t stream);
int ob_radial_divergence(const float* xyz, const int32_t* faces, int n_faces, int n_vertices,
                         const double* tangent_angles, const double* transport_angles, const double* fields, int source,
                         const float* cot, const int32_t* corner_offsets, const int32_t* corner_slots,
                         double* corner_scratch, double* divergence, ob_stream_t stream);
int ob_log_map_fields(const double* fields, const double* distance, int source, int n_vertices, float* out,
                      ob_stream_t stream);

/* ---- a12: the marched settled solve --------------------------------------------------------
 * Replaces ordito/linalg.py:2765 _march_settled (kernels/linalg.py:1229-1545): x = A^-1 rhs for
 * one column, band by band outward from rhs's support, every entry to its own relative
 * precision -- the settled solve's fallback where the operator's factorisation is refused. Bands
 * grow breadth first from the finished rows; each band system (Dirichlet data from the finished
 * neighbours, zero beyond, scaled so its front is O(1)) is solved by float64 CG to a relative
 * residual of 1e-14; rows within e^14 of the band's peak and e^16 above its outer layer are
 * finished. x is overwritten (its input is ignored). info[0..2] (may be NULL) = bands, CG rounds,
 * band rows solved. Synchronises the stream (the loop reads each band's size back). */
int ob_march_solve(int n, const int32_t* offsets, const int32_t* columns, const double* values,
                   const double* rhs, double* x, long long* info, ob_stream_t stream);

/* ---- f4: the intrinsic tufted cover (use_robust at method="potpourri3d") --------------------
 * ob_cover_build replaces ordito/heat.py:5084 _tufted_intrinsic_delaunay (kernels/heat.py:749-1130:
 * tufted_cover, glue_nonmanifold_cover_edges, length_sum_and_violation, mollify_cover_lengths,
 * cover_flip_candidates / _commit / _fixup). From the mesh's operator pattern (ob_pattern_build:
 * its runs give each edge's halfedges) and its float32 positions: cover_faces[6 F] (cover face
 * f < F the front copy of face f, F + f its back copy (c0, c2, c1)), lengths[6 F] (float64, slot
 * 3 g + e the edge of cover face g opposite its corner e) and twin[6 F], mollified by
 * max(0, worst violation + epsilon_mollify * mean front length) and flipped to intrinsic Delaunay
 * (an edge flips while its two facing half-cotangents sum below -epsilon_delaunay) in rounds of
 * independent sets -- the lowest candidate of each face claims it -- until a round flips nothing
 * or max_rounds ran; *rounds (may be NULL) = rounds run. Every float64 step rounds once (no fused
 * multiply-adds). Synchronises the stream (each round's flip count is read back). An edge of more
 * than 64 faces is rejected (OB_ERR_INVALID).
 * ob_cover_face_terms replaces kernels/heat.py:1133 cover_face_terms: cot[3 n_cover] the float64
 * half-cotangents, area_sums[V] each vertex's corner areas (Heron, in float64) summed in ascending
 * corner order (corner index of cover_faces from ob_corner_index), length_sums[2] (device) the sum
 * and count of every slot's length -- the mean cover edge of the default time step.
 * ob_cover_divergence replaces kernels/heat.py:1154 cover_unit_gradient_divergence: out[V][k] =
 * div of the unit gradient of u[V][k] on the cover, each face laid out in the plane from its
 * lengths, every vertex's corner terms summed in ascending corner order. */
int ob_cover_build(const int32_t* offsets, const int32_t* columns, const int32_t* run_start,
                   const uint64_t* keys, int n_keys, const int32_t* order, int n_vertices,
                   const float* xyz, const int32_t* faces, int n_faces, double epsilon_mollify,
                   double epsilon_delaunay, int max_rounds, int32_t* cover_faces, double* lengths,
                   int32_t* twin, int32_t* rounds, ob_stream_t stream);
int ob_cover_face_terms(const int32_t* cover_faces, const double* lengths, int n_cover, int n_vertices,
                        const int32_t* corner_offsets, const int32_t* corner_slots, double* cot,
                        double* area_sums, double* length_sums, ob_stream_t stream);
int ob_cover_divergence(const int32_t* cover_faces, const double* lengths, const double* cot, int n_vertices,
                        const int32_t* corner_offsets, const int32_t* corner_slots, const double* u,
                        int n_columns, double* out, ob_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* ORDITO_B200_H */
