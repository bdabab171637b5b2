// a7/a9: preconditioned conjugate gradient over one CSR operator and n_columns right-hand sides.
//
// The iteration is Chronopoulos-Gear CG (the form ordito/kernels/algorithms/conjugate_gradient.py
// :397-838 uses): a round is one mat-vec that also reduces the round's three dot products
// (gamma = r.u, delta = w.u, r.r) and one fused update (p, s, x, r and the Jacobi apply), with
// alpha and beta recovered from the dots. The dots are reduced per block in a fixed tree and
// folded in block order by the last block to finish, so every run gives the same bits, and that
// block derives the round's scalars once for everyone. The loop runs on the device: a CUDA graph
// whose conditional WHILE node replays a body of `rounds_per_body` rounds and one decision kernel
// (the settle check of linalg.solve_spd_settled, ordito/linalg.py:2490, or the residual test of
// solve_spd, :1356), so a solve is one graph launch with no host round trip per round.
//
// Layout: vectors hold n_columns interleaved columns, [row][column], so the threads of one row's
// columns gather the same neighbours' contiguous column blocks (coalesced) while the row's
// indices and values are broadcast. The column count is padded to a power of two (<= 256); pad
// columns have a zero right-hand side and never step. The iteration's mat-vecs read a sliced-ELL
// copy of the operator the solver builds from the CSR arrays it is given (slices of 32 rows, each
// as wide as its longest row, column-major within the slice): the 32 rows a warp serves at one
// column read an entry index's values and columns as one contiguous 256- and 128-byte access,
// where the CSR rows' entries would be 32 scattered ones.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ob_internal.cuh"
#include "ob_scratch.cuh"

namespace ob {
namespace {

constexpr int kThreads = 256;
constexpr int kChebyshevDegree = 12;  // ordito/linalg.py:5368 CHEBYSHEV_DEGREE
constexpr double kChebyshevInterval = 80.0;  // :5369 CHEBYSHEV_INTERVAL
constexpr double kIntervalCap = 0.5;         // :5360 SQUARED_LAPLACIAN_INTERVAL_CAP

// Device-side loop state of one solver.
struct LoopState {
    int round;        // rounds run (the round index the next mat-vec measures)
    int iterations;   // rounds in which some column stepped
    int done;         // set when no column stepped or the cap was reached
    int status;       // OB_STATUS_*
    int settle_checks_unused;
};

// Settle monitor (ordito/kernels/algorithms/conjugate_gradient.py:1490-1580).
struct SettleState {
    double change;       // max relative change since the last check
    double reached;      // count of non-zero entries
    double previous;     // reached count + 1 at the last change
    double reach_check;  // check index at the last change
    double checks;       // checks so far
};

struct ColumnScalars {
    double gamma_old, alpha_old, atol_sq, alpha, beta, rr, rr0;
    int step;
    int pad;
};

// Fixed-tree reduction of per-thread values grouped by column (thread t holds column t % k).
// On return sh[c] (c < k) holds column c's block total. k divides blockDim.x (power of two).
__device__ __forceinline__ void column_tree(double* sh, int k) {
    for (int s = blockDim.x >> 1; s >= k; s >>= 1) {
        __syncthreads();
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    }
    __syncthreads();
}

__device__ __forceinline__ void column_tree_max(double* sh, int k) {
    for (int s = blockDim.x >> 1; s >= k; s >>= 1) {
        __syncthreads();
        if ((int)threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
    }
    __syncthreads();
}

template <typename V>
__device__ __forceinline__ double row_dot(const int* __restrict__ offsets,
                                          const int* __restrict__ columns,
                                          const V* __restrict__ values,
                                          const double* __restrict__ x, int row, int k, int c) {
    double acc = 0.0;
    const int end = offsets[row + 1];
    for (int j = offsets[row]; j < end; ++j)
        acc = fma((double)values[j], x[(size_t)columns[j] * k + c], acc);
    return acc;
}

// Sliced ELL: slice s holds rows [32 s, 32 s + 32); entry j of its row l sits at
// start[s] + 32 j + l, start[s + 1] - start[s] = 32 x the slice's widest row. Padding entries
// name the row itself with a zero value, so a row's sum is the CSR row's, in the same order,
// followed by exact zeros.
constexpr int kSlice = 32;

template <typename V>
struct Sell {
    const long long* __restrict__ start;
    const int* __restrict__ columns;
    const V* __restrict__ values;
    // The copy is larger than half the L2: its columns and values are read with the evict-first
    // hint, so the gathered vector stays in L2 (2.6 M-vertex torus: 69.4 -> 64.2 us a mat-vec). A
    // smaller copy stays in L2 itself across the solver's rounds, which the hint would undo.
    int stream;
};

template <typename V>
__device__ __forceinline__ double sell_row_dot(const Sell<V> A, const double* __restrict__ x, int row,
                                               int k, int c) {
    const int slice = row / kSlice, lane = row % kSlice;
    const long long base = A.start[slice];
    const int width = (int)((A.start[slice + 1] - base) / kSlice);
    const int* __restrict__ cols = A.columns + base + lane;
    const V* __restrict__ vals = A.values + base + lane;
    double acc = 0.0;
    if (A.stream) {
#pragma unroll 4
        for (int j = 0; j < width; ++j)
            acc = fma((double)__ldcs(vals + (size_t)kSlice * j), x[(size_t)__ldcs(cols + (size_t)kSlice * j) * k + c],
                      acc);
    } else {
#pragma unroll 4
        for (int j = 0; j < width; ++j)
            acc = fma((double)__ldg(vals + (size_t)kSlice * j), x[(size_t)__ldg(cols + (size_t)kSlice * j) * k + c],
                      acc);
    }
    return acc;
}

// 32 x the widest row of each slice (entry n_slices: 0, for the scan's total).
__global__ void slice_width_kernel(int n, int n_slices, const int* __restrict__ offsets,
                                   long long* __restrict__ width) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s > n_slices) return;
    int w = 0;
    if (s < n_slices) {
        const int end = min(n, (s + 1) * kSlice);
        for (int r = s * kSlice; r < end; ++r) w = max(w, offsets[r + 1] - offsets[r]);
    }
    width[s] = (long long)w * kSlice;
}

// Writes the sliced-ELL copy (and its float32 values when `values32` is given), a thread a row.
__global__ void slice_fill_kernel(int n, const int* __restrict__ offsets, const int* __restrict__ columns,
                                  const double* __restrict__ values, const long long* __restrict__ start,
                                  int* __restrict__ sell_columns, double* __restrict__ sell_values,
                                  float* __restrict__ sell_values32) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    const int slice = row / kSlice, lane = row % kSlice;
    const long long base = start[slice];
    const int width = (int)((start[slice + 1] - base) / kSlice);
    const int o = offsets[row], d = offsets[row + 1] - o;
    for (int j = 0; j < width; ++j) {
        const long long at = base + (long long)kSlice * j + lane;
        const int col = j < d ? columns[o + j] : row;
        const double v = j < d ? values[o + j] : 0.0;
        sell_columns[at] = col;
        sell_values[at] = v;
        if (sell_values32) sell_values32[at] = (float)v;
    }
}

// Jacobi setup (ordito/kernels/linalg.py jacobi_dominance_bound and chebyshev_steps :1530-1583):
// D^-1 (0 for a row without a diagonal entry), the rows' largest Gershgorin ratio
// sum_{j != i} |A_ij| / |A_ii|, and the Chebyshev steps fitted to it by the last block.
__global__ void jacobi_setup_kernel(int n, const int* __restrict__ offsets,
                                    const int* __restrict__ columns,
                                    const double* __restrict__ values,
                                    double* __restrict__ inv_diag, double* __restrict__ maxima,
                                    unsigned int* counter, int n_steps,
                                    double4* __restrict__ steps) {
    __shared__ double scratch[32];
    __shared__ int last;
    double ratio = -INFINITY;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double diag = 0.0, off = 0.0;
        for (int j = offsets[i]; j < offsets[i + 1]; ++j) {
            if (columns[j] == i)
                diag = values[j];
            else
                off += fabs(values[j]);
        }
        inv_diag[i] = diag != 0.0 ? 1.0 / diag : 0.0;
        if (diag != 0.0) ratio = fmax(ratio, off / fabs(diag));
    }
    const double bm = block_max(ratio, scratch, -(double)INFINITY);
    if (threadIdx.x == 0) maxima[blockIdx.x] = bm;
    if (!last_block_arrived(counter, &last)) return;
    if (threadIdx.x != 0) return;
    double maximum = -INFINITY;
    for (int b = 0; b < (int)gridDim.x; ++b) maximum = fmax(maximum, __ldcg(&maxima[b]));
    const double relative = fmin(kChebyshevInterval / (double)max(n, 1), kIntervalCap);
    const double dominance = fmax(maximum, 1e-3);
    const double lower = fmax(relative, 1.0 - dominance);
    const double upper = 1.0 + dominance;
    const double theta = 0.5 * (upper + lower), delta = 0.5 * (upper - lower);
    const double sigma = theta / delta;
    double rho = 1.0 / sigma;
    for (int index = 0; index < n_steps; ++index) {
        const double rho_next = 1.0 / (2.0 * sigma - rho);
        double scale = 1.0, previous_scale = 1.0;
        if (index == 0) {
            scale = 1.0 / theta;
            previous_scale = 0.0;
        } else if (index == 1) {
            previous_scale = 1.0 / theta;
        }
        steps[index] = make_double4(scale, previous_scale, rho_next * rho, 2.0 * rho_next / delta);
        rho = rho_next;
    }
}

// r = b - A x (float64 values), u = D^-1 r (Jacobi) or scaled = D^-1 r (polynomial input).
__global__ void initial_residual_kernel(int n, int k, const int* __restrict__ offsets,
                                        const int* __restrict__ columns,
                                        const double* __restrict__ values,
                                        const double* __restrict__ b, const double* __restrict__ x,
                                        const double* __restrict__ inv_diag,
                                        double* __restrict__ r, double* __restrict__ u) {
    const long long total = (long long)n * k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(t / k), c = (int)(t % k);
        const double ri = b[t] - row_dot(offsets, columns, values, x, row, k, c);
        r[t] = ri;
        u[t] = inv_diag[row] * ri;
    }
}

// Per-column |b|^2 into scalars (rr0, atol_sq) and the loop state reset.
__global__ void reset_kernel(int n, int k, int k_live, const double* __restrict__ b, double tol,
                             double* __restrict__ partials, unsigned int* counter,
                             ColumnScalars* __restrict__ scalars, LoopState* state,
                             SettleState* settle) {
    __shared__ double sh[kThreads];
    __shared__ int last;
    const int c = threadIdx.x % k;
    double acc = 0.0;
    const long long total = (long long)n * k;
    const long long stride = (long long)gridDim.x * blockDim.x;  // a multiple of k
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += stride) {
        const double v = b[t];
        acc = fma(v, v, acc);
    }
    sh[threadIdx.x] = acc;
    column_tree(sh, k);
    if ((int)threadIdx.x < k) partials[(size_t)blockIdx.x * k + threadIdx.x] = sh[threadIdx.x];
    if (!last_block_arrived(counter, &last)) return;
    const int groups = blockDim.x / k, g = threadIdx.x / k;
    double sum = 0.0;
    for (int bx = g; bx < (int)gridDim.x; bx += groups) sum += __ldcg(&partials[(size_t)bx * k + c]);
    sh[threadIdx.x] = sum;
    column_tree(sh, k);
    if ((int)threadIdx.x < k) {
        ColumnScalars s;
        s.rr0 = sh[threadIdx.x];
        s.atol_sq = (threadIdx.x < (unsigned)k_live) ? tol * tol * s.rr0 : INFINITY;
        s.gamma_old = INFINITY;
        s.alpha_old = 1.0;
        s.alpha = s.beta = 0.0;
        s.rr = s.rr0;
        s.step = 0;
        s.pad = 0;
        scalars[threadIdx.x] = s;
    }
    if (threadIdx.x == 0) {
        state->round = 0;
        state->iterations = 0;
        state->done = 0;
        state->status = OB_STATUS_CAPPED;
        settle->change = 0.0;
        settle->reached = 0.0;
        settle->previous = 0.0;
        settle->reach_check = 0.0;
        settle->checks = 0.0;
    }
}

// The first node of a round: w = A u and the block partials of (r.u, w.u, r.r) per column; the last
// block folds them per column in block order and derives (alpha, beta, step) (cg_step_scalars,
// conjugate_gradient.py:549-579), then counts the round (cg_close_round :628-669).
template <typename V>
__global__ void __launch_bounds__(kThreads, 8) matvec_dots_kernel(int n, int k, const Sell<V> A,
                                   const double* __restrict__ r, const double* __restrict__ u,
                                   double* __restrict__ w, double* __restrict__ partials,
                                   unsigned int* counter, ColumnScalars* __restrict__ scalars,
                                   LoopState* state, int maxiter) {
    __shared__ double sg[kThreads], sd[kThreads], sr[kThreads];
    __shared__ int last;
    if (state->done) {
        // The loop is over: the rounds left in this body change nothing.
        if (blockIdx.x == 0 && (int)threadIdx.x < k) scalars[threadIdx.x].step = 0;
        return;
    }
    const int c = threadIdx.x % k;
    double ag = 0.0, ad = 0.0, ar = 0.0;
    const long long total = (long long)n * k;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += stride) {
        const int row = (int)(t / k);
        const double wi = sell_row_dot(A, u, row, k, c);
        w[t] = wi;
        const double ri = r[t], ui = u[t];
        ag = fma(ri, ui, ag);
        ad = fma(wi, ui, ad);
        ar = fma(ri, ri, ar);
    }
    sg[threadIdx.x] = ag;
    sd[threadIdx.x] = ad;
    sr[threadIdx.x] = ar;
    for (int s = blockDim.x >> 1; s >= k; s >>= 1) {
        __syncthreads();
        if ((int)threadIdx.x < s) {
            sg[threadIdx.x] += sg[threadIdx.x + s];
            sd[threadIdx.x] += sd[threadIdx.x + s];
            sr[threadIdx.x] += sr[threadIdx.x + s];
        }
    }
    __syncthreads();
    if ((int)threadIdx.x < k) {
        double* p = partials + ((size_t)blockIdx.x * k + threadIdx.x) * 3;
        p[0] = sg[threadIdx.x];
        p[1] = sd[threadIdx.x];
        p[2] = sr[threadIdx.x];
    }
    if (!last_block_arrived(counter, &last)) return;
    const int groups = blockDim.x / k, g = threadIdx.x / k;
    double fg = 0.0, fd = 0.0, fr = 0.0;
    for (int bx = g; bx < (int)gridDim.x; bx += groups) {
        const double* p = partials + ((size_t)bx * k + c) * 3;
        fg += __ldcg(p);
        fd += __ldcg(p + 1);
        fr += __ldcg(p + 2);
    }
    sg[threadIdx.x] = fg;
    sd[threadIdx.x] = fd;
    sr[threadIdx.x] = fr;
    for (int s = blockDim.x >> 1; s >= k; s >>= 1) {
        __syncthreads();
        if ((int)threadIdx.x < s) {
            sg[threadIdx.x] += sg[threadIdx.x + s];
            sd[threadIdx.x] += sd[threadIdx.x + s];
            sr[threadIdx.x] += sr[threadIdx.x + s];
        }
    }
    __syncthreads();
    __shared__ int any_step, any_nan;
    if (threadIdx.x == 0) {
        any_step = 0;
        any_nan = 0;
    }
    __syncthreads();
    const int round_index = state->round;
    if ((int)threadIdx.x < k) {
        ColumnScalars s = scalars[threadIdx.x];
        const double gamma = sg[threadIdx.x], delta = sd[threadIdx.x], rr = sr[threadIdx.x];
        s.rr = rr;
        s.step = 0;
        s.alpha = 0.0;
        s.beta = 0.0;
        if (rr > s.atol_sq && round_index <= maxiter && gamma != 0.0) {
            const double beta = gamma / s.gamma_old;
            const double denominator = delta - beta * gamma / s.alpha_old;
            if (denominator != 0.0) {
                s.alpha = gamma / denominator;
                s.beta = beta;
                s.step = 1;
                s.gamma_old = gamma;
                s.alpha_old = s.alpha;
            }
        }
        if (!(rr == rr)) atomicOr(&any_nan, 1);
        if (s.step) atomicOr(&any_step, 1);
        scalars[threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        state->round = round_index + 1;
        state->iterations += any_step;
        if (!any_step || round_index >= maxiter) {
            state->done = 1;
            state->status = any_nan ? OB_STATUS_NONFINITE
                            : (!any_step && round_index <= maxiter) ? OB_STATUS_CONVERGED
                                                                     : OB_STATUS_CAPPED;
        }
    }
}

// The second node: p = u + beta p, s = w + beta s, x += alpha p, r -= alpha s and the Jacobi apply
// D^-1 r into `scaled` (which is u itself under Jacobi, the polynomial's input under Chebyshev)
// for every column that stepped (conjugate_gradient.py:797-838, cg_advance :413).
__global__ void __launch_bounds__(kThreads, 8) update_kernel(int n, int k, const ColumnScalars* __restrict__ scalars,
                              const double* __restrict__ inv_diag, const double* __restrict__ w,
                              const double* u, double* __restrict__ p, double* __restrict__ s,
                              double* __restrict__ r, double* __restrict__ x, double* scaled) {
    const long long total = (long long)n * k;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int c = threadIdx.x % k;
    const ColumnScalars sc = scalars[c];
    if (!sc.step) return;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += stride) {
        const int row = (int)(t / k);
        const double pn = fma(sc.beta, p[t], u[t]);
        const double sn = fma(sc.beta, s[t], w[t]);
        p[t] = pn;
        s[t] = sn;
        x[t] = fma(sc.alpha, pn, x[t]);
        const double rn = fma(-sc.alpha, sn, r[t]);
        r[t] = rn;
        scaled[t] = inv_diag[row] * rn;
    }
}

// One step of the Jacobi-Chebyshev polynomial (ordito/kernels/algorithms/multigrid.py:926-1033,
// chebyshev_update / chebyshev_step): out = s x + momentum (s x - s_prev x_prev)
// + step (source - s D^-1 A x), steps[index] = (s, s_prev, momentum, step). `out` may alias
// `x_prev` but not `x`.
template <typename V>
__global__ void chebyshev_step_kernel(int n, int k, const Sell<V> A,
                                      const double* __restrict__ inv_diag,
                                      const double4* __restrict__ steps, int index,
                                      const double* __restrict__ source,
                                      const double* __restrict__ x, const double* x_prev,
                                      double* out, const LoopState* state) {
    if (state->done) return;
    const double4 st = steps[index];
    const long long total = (long long)n * k;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int c = threadIdx.x % k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += stride) {
        const int row = (int)(t / k);
        const double ax = sell_row_dot(A, x, row, k, c) * inv_diag[row];
        const double current = st.x * x[t];
        out[t] = current + st.z * (current - st.y * x_prev[t]) + st.w * (source[t] - st.x * ax);
    }
}

// The settle check (cg_settle_change / cg_settle_verdict, conjugate_gradient.py:1500-1580): the
// largest |x - previous| / |x| over non-zero entries and their count, over every column; previous
// advances to x. The last block applies the verdict.
__global__ void __launch_bounds__(kThreads, 8) settle_kernel(long long total, const double* __restrict__ x,
                              double* __restrict__ previous, double2* __restrict__ partials,
                              unsigned int* counter, SettleState* settle, LoopState* state,
                              int check_rounds, double change_tolerance, int settle_rounds) {
    __shared__ double scratch[32];
    __shared__ int last;
    if (state->done) return;
    double change = 0.0, reached = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const double v = x[t];
        if (v != 0.0) {
            change = fmax(change, fabs(v - previous[t]) / fabs(v));
            reached += 1.0;
        }
        previous[t] = v;
    }
    const double bm = block_max(change, scratch, 0.0);
    const double bs = block_sum(reached, scratch);
    if (threadIdx.x == 0) partials[blockIdx.x] = make_double2(bm, bs);
    if (!last_block_arrived(counter, &last)) return;
    if (threadIdx.x != 0) return;
    double m = 0.0, cnt = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) {
        const double2 p = __ldcg(&partials[b]);
        m = fmax(m, p.x);
        cnt += p.y;
    }
    const double checks = settle->checks + 1.0;
    settle->checks = checks;
    const double count = cnt + 1.0;
    if (count != settle->previous) {
        settle->previous = count;
        settle->reach_check = checks;
        return;
    }
    const double idle = (checks - settle->reach_check) * (double)check_rounds;
    if (m < change_tolerance || idle >= (double)settle_rounds) {
        state->done = 1;
        state->status = (m < change_tolerance) ? OB_STATUS_SETTLED : OB_STATUS_SETTLE_BOUND;
    }
}

// Clears the step flags once the loop is over (the rounds left in a body then change nothing),
// and hands the loop condition to the graph's WHILE node.
__global__ void decide_kernel(LoopState* state, ColumnScalars* scalars, int k,
                              cudaGraphConditionalHandle handle) {
    const int done = state->done;
    if (done)
        for (int c = threadIdx.x; c < k; c += blockDim.x) scalars[c].step = 0;
    if (threadIdx.x == 0) cudaGraphSetConditional(handle, done ? 0u : 1u);
}

// y = A x over n_columns interleaved columns (float64).
__global__ void spmv_kernel(int n, int k, const int* __restrict__ offsets,
                            const int* __restrict__ columns, const double* __restrict__ values,
                            const double* __restrict__ x, double* __restrict__ y) {
    const long long total = (long long)n * k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x)
        y[t] = row_dot(offsets, columns, values, x, (int)(t / k), k, (int)(t % k));
}

// Componentwise backward error (Oettli-Prager; ordito/kernels/linalg.py:1167-1210): flag rows
// with |b - A x|_i > tol (|A| |x| + |b|)_i, or a NaN.
__global__ void backward_error_kernel(int n, int k, const int* __restrict__ offsets,
                                      const int* __restrict__ columns,
                                      const double* __restrict__ values,
                                      const double* __restrict__ x, const double* __restrict__ b,
                                      double tol, int* __restrict__ flag) {
    const long long total = (long long)n * k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(t / k), c = (int)(t % k);
        double ax = 0.0, scale = 0.0;
        for (int j = offsets[row]; j < offsets[row + 1]; ++j) {
            const double a = values[j], xv = x[(size_t)columns[j] * k + c];
            ax = fma(a, xv, ax);
            scale = fma(fabs(a), fabs(xv), scale);
        }
        const double residual = fabs(b[t] - ax);
        scale += fabs(b[t]);
        if (!(residual <= tol * scale)) atomicOr(flag, 1);
    }
}

int next_pow2(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

struct Solver {
    int n = 0, k_live = 0, k = 0, precond = 0, narrow = 0;
    long long nnz = 0;
    const int* offsets = nullptr;
    const int* columns = nullptr;
    const double* values = nullptr;
    // The sliced-ELL copy the iteration's mat-vecs read (its float32 values when narrow), grown
    // when a rebound operator's slices need more entries than it holds.
    int n_slices = 0;
    long long* sell_start = nullptr;
    int* sell_columns = nullptr;
    double* sell_values = nullptr;
    float* sell_values32 = nullptr;
    long long sell_capacity = 0;
    long long sell_entries = 0;  // the current operator's (padding included)
    double *inv_diag = nullptr, *b = nullptr, *x = nullptr, *r = nullptr, *u = nullptr,
           *w = nullptr, *p = nullptr, *s = nullptr, *scaled = nullptr, *t0 = nullptr,
           *t1 = nullptr, *previous = nullptr, *partials = nullptr, *maxima = nullptr;
    double2* settle_partials = nullptr;
    double4* steps = nullptr;
    ColumnScalars* scalars = nullptr;
    LoopState* state = nullptr;
    SettleState* settle = nullptr;
    unsigned int* counters = nullptr;  // [0] matvec, [1] settle, [2] reset, [3] setup
    LoopState* host_state = nullptr;   // pinned
    ColumnScalars* host_scalars = nullptr;
    int blocks = 0;
    cudaStream_t capture = nullptr;
    // Cached loop graphs: key = (settle?, rounds per body, maxiter, params).
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    cudaGraph_t graph[2] = {nullptr, nullptr};
    int exec_rounds[2] = {0, 0};
    int exec_maxiter[2] = {0, 0};
    double exec_change[2] = {0.0, 0.0};
    int exec_settle[2] = {0, 0};
    std::vector<void*> owned;
};

void release_sell(Solver* S) {
    for (void* p : {(void*)S->sell_columns, (void*)S->sell_values, (void*)S->sell_values32})
        if (p) cudaFree(p);
    S->sell_columns = nullptr;
    S->sell_values = nullptr;
    S->sell_values32 = nullptr;
    S->sell_capacity = 0;
}

void drop_graphs(Solver* S) {
    for (int i = 0; i < 2; ++i) {
        if (S->exec[i]) cudaGraphExecDestroy(S->exec[i]);
        if (S->graph[i]) cudaGraphDestroy(S->graph[i]);
        S->exec[i] = nullptr;
        S->graph[i] = nullptr;
    }
}

// Builds the sliced-ELL copy of the solver's CSR operator: slice widths, their scan (read back
// once, to size the copy), the fill. A copy that must grow is reallocated, and the recorded loops
// that name the old one are dropped (rebuilt at the next solve).
int build_sell(Solver* S, cudaStream_t stream) {
    const int n_slices = S->n_slices;
    {
        Scratch scratch(stream);
        long long* width = scratch.take<long long>((size_t)n_slices + 1);
        size_t bytes = 0;
        OB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, width, S->sell_start, n_slices + 1, stream));
        void* temp = scratch.take<unsigned char>(bytes);
        if (int st = scratch.commit()) return st;
        slice_width_kernel<<<ceil_div(n_slices + 1, kThreads), kThreads, 0, stream>>>(S->n, n_slices, S->offsets,
                                                                                       width);
        OB_CHECK_LAUNCH("pcg slice widths");
        OB_CUDA(cub::DeviceScan::ExclusiveSum(temp, bytes, width, S->sell_start, n_slices + 1, stream));
    }
    long long total = 0;
    OB_CUDA(cudaMemcpyAsync(&total, S->sell_start + n_slices, sizeof(long long), cudaMemcpyDeviceToHost,
                            stream));
    OB_CUDA(cudaStreamSynchronize(stream));
    if (total > S->sell_capacity) {
        drop_graphs(S);
        release_sell(S);
        const size_t entries = (size_t)std::max(total, 1LL);
        cudaError_t e = pool_malloc((void**)&S->sell_columns, sizeof(int) * entries, stream);
        if (e == cudaSuccess) e = pool_malloc((void**)&S->sell_values, sizeof(double) * entries, stream);
        if (e == cudaSuccess && S->narrow)
            e = pool_malloc((void**)&S->sell_values32, sizeof(float) * entries, stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            release_sell(S);
            return cuda_status(e, "pcg sliced-ELL copy");
        }
        S->sell_capacity = total;
    }
    S->sell_entries = total;
    slice_fill_kernel<<<ceil_div(S->n, kThreads), kThreads, 0, stream>>>(
        S->n, S->offsets, S->columns, S->values, S->sell_start, S->sell_columns, S->sell_values,
        S->narrow ? S->sell_values32 : nullptr);
    OB_CHECK_LAUNCH("pcg slice fill");
    return OB_OK;
}

// Half the L2 (126 MB on B200): a sliced-ELL copy above it is streamed (Sell::stream).
constexpr long long kStreamBytes = 63LL << 20;
Sell<double> sell64(const Solver* S) {
    return Sell<double>{S->sell_start, S->sell_columns, S->sell_values, S->sell_entries * 12 > kStreamBytes};
}
Sell<float> sell32(const Solver* S) {
    return Sell<float>{S->sell_start, S->sell_columns, S->sell_values32, S->sell_entries * 8 > kStreamBytes};
}

// Copies an operator of the solver's shape into its own arrays and derives what the iteration
// reads from it: the inverse diagonal, the Chebyshev steps and the sliced-ELL copy.
int bind_operator(Solver* S, const int* offsets, const int* columns, const double* values,
                  cudaStream_t stream) {
    const int n = S->n;
    const long long nnz = S->nnz;
    OB_CUDA(cudaMemcpyAsync(const_cast<int*>(S->offsets), offsets, sizeof(int) * (size_t)(n + 1),
                            cudaMemcpyDeviceToDevice, stream));
    if (nnz > 0) {
        OB_CUDA(cudaMemcpyAsync(const_cast<int*>(S->columns), columns, sizeof(int) * (size_t)nnz,
                                cudaMemcpyDeviceToDevice, stream));
        OB_CUDA(cudaMemcpyAsync(const_cast<double*>(S->values), values, sizeof(double) * (size_t)nnz,
                                cudaMemcpyDeviceToDevice, stream));
    }
    const int setup_blocks = std::max(1, std::min(ceil_div(n, kThreads), 4 * sm_count()));
    jacobi_setup_kernel<<<setup_blocks, kThreads, 0, stream>>>(
        n, S->offsets, S->columns, S->values, S->inv_diag, S->maxima, S->counters + 3,
        kChebyshevDegree - 1, S->steps);
    OB_CHECK_LAUNCH("pcg setup");
    return build_sell(S, stream);
}

int solver_alloc(Solver* S, void** out, size_t bytes, cudaStream_t stream) {
    OB_CUDA(pool_malloc(out, bytes == 0 ? 8 : bytes, stream));
    S->owned.push_back(*out);
    return OB_OK;
}

void solver_release(Solver* S) {
    drop_graphs(S);
    release_sell(S);
    for (void* p : S->owned) cudaFree(p);
    if (S->host_state) cudaFreeHost(S->host_state);
    if (S->host_scalars) cudaFreeHost(S->host_scalars);
    if (S->capture) cudaStreamDestroy(S->capture);
    delete S;
}

// Enqueues one round (mat-vec with dots, update, and the polynomial when preconditioned by it).
int enqueue_round(Solver* S, cudaStream_t stream, int maxiter) {
    const int B = S->blocks;
    if (S->narrow)
        matvec_dots_kernel<float><<<B, kThreads, 0, stream>>>(
            S->n, S->k, sell32(S), S->r, S->u, S->w, S->partials, S->counters, S->scalars, S->state,
            maxiter);
    else
        matvec_dots_kernel<double><<<B, kThreads, 0, stream>>>(
            S->n, S->k, sell64(S), S->r, S->u, S->w, S->partials, S->counters, S->scalars, S->state,
            maxiter);
    OB_CHECK_LAUNCH("matvec_dots");
    double* target = (S->precond == 1) ? S->scaled : S->u;
    update_kernel<<<B, kThreads, 0, stream>>>(S->n, S->k, S->scalars, S->inv_diag, S->w, S->u,
                                              S->p, S->s, S->r, S->x, target);
    OB_CHECK_LAUNCH("update");
    if (S->precond == 1) {
        const int n_steps = kChebyshevDegree - 1;
        const double* in = S->scaled;
        const double* prev = S->scaled;
        double* bufs[2] = {S->t0, S->t1};
        for (int index = 0; index < n_steps; ++index) {
            double* out = (index == n_steps - 1) ? S->u : bufs[index & 1];
            if (S->narrow)
                chebyshev_step_kernel<float><<<B, kThreads, 0, stream>>>(
                    S->n, S->k, sell32(S), S->inv_diag, S->steps, index, S->scaled, in, prev, out,
                    S->state);
            else
                chebyshev_step_kernel<double><<<B, kThreads, 0, stream>>>(
                    S->n, S->k, sell64(S), S->inv_diag, S->steps, index, S->scaled, in, prev, out,
                    S->state);
            OB_CHECK_LAUNCH("chebyshev_step");
            prev = in;
            in = out;
        }
    }
    return OB_OK;
}

// The polynomial apply u = p(D^-1 A) scaled outside the loop (the initial preconditioned residual).
int enqueue_polynomial(Solver* S, cudaStream_t stream) {
    const int B = S->blocks;
    const int n_steps = kChebyshevDegree - 1;
    const double* in = S->scaled;
    const double* prev = S->scaled;
    double* bufs[2] = {S->t0, S->t1};
    for (int index = 0; index < n_steps; ++index) {
        double* out = (index == n_steps - 1) ? S->u : bufs[index & 1];
        if (S->narrow)
            chebyshev_step_kernel<float><<<B, kThreads, 0, stream>>>(
                S->n, S->k, sell32(S), S->inv_diag, S->steps, index, S->scaled, in, prev, out,
                S->state);
        else
            chebyshev_step_kernel<double><<<B, kThreads, 0, stream>>>(
                S->n, S->k, sell64(S), S->inv_diag, S->steps, index, S->scaled, in, prev, out,
                S->state);
        OB_CHECK_LAUNCH("chebyshev_step");
        prev = in;
        in = out;
    }
    return OB_OK;
}

// Builds (or reuses) the loop graph: a WHILE node whose body is `rounds` rounds, the settle check
// (settle mode) and the decision kernel.
int loop_graph(Solver* S, int mode, int rounds, int maxiter, int check_rounds, double change_tol,
               int settle_rounds) {
    if (S->exec[mode] && S->exec_rounds[mode] == rounds && S->exec_maxiter[mode] == maxiter &&
        S->exec_change[mode] == change_tol && S->exec_settle[mode] == settle_rounds)
        return OB_OK;
    if (S->exec[mode]) {
        cudaGraphExecDestroy(S->exec[mode]);
        cudaGraphDestroy(S->graph[mode]);
        S->exec[mode] = nullptr;
        S->graph[mode] = nullptr;
    }
    cudaGraph_t graph;
    OB_CUDA(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle handle;
    cudaError_t e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_status(e, "cudaGraphConditionalHandleCreate");
    }
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, graph, nullptr, 0, &params);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_status(e, "cudaGraphAddNode(conditional)");
    }
    cudaGraph_t body = params.conditional.phGraph_out[0];
    std::lock_guard<std::recursive_mutex> guard(capture_mutex());
    e = cudaStreamBeginCaptureToGraph(S->capture, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_status(e, "cudaStreamBeginCaptureToGraph");
    }
    int st = OB_OK;
    suppress_counting(1);
    for (int i = 0; i < rounds && st == OB_OK; ++i) st = enqueue_round(S, S->capture, maxiter);
    if (st == OB_OK && mode == 1) {
        const long long total = (long long)S->n * S->k;
        settle_kernel<<<S->blocks, kThreads, 0, S->capture>>>(
            total, S->x, S->previous, S->settle_partials, S->counters + 1, S->settle, S->state,
            check_rounds, change_tol, settle_rounds);
        count_launch();
    }
    if (st == OB_OK) {
        decide_kernel<<<1, 32, 0, S->capture>>>(S->state, S->scalars, S->k, handle);
        count_launch();
    }
    suppress_counting(-1);
    cudaGraph_t captured;
    e = cudaStreamEndCapture(S->capture, &captured);
    if (st != OB_OK || e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return st != OB_OK ? st : cuda_status(e, "cudaStreamEndCapture");
    }
    cudaGraphExec_t exec;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_status(e, "cudaGraphInstantiate");
    }
    S->graph[mode] = graph;
    S->exec[mode] = exec;
    S->exec_rounds[mode] = rounds;
    S->exec_maxiter[mode] = maxiter;
    S->exec_change[mode] = change_tol;
    S->exec_settle[mode] = settle_rounds;
    return OB_OK;
}

// Copies rhs / x in, resets the state and forms r, u; tol is the relative residual tolerance.
int start_solve(Solver* S, const double* rhs, const double* x, double tol, cudaStream_t stream) {
    const size_t live = sizeof(double) * (size_t)S->n * S->k;
    if (S->k == S->k_live) {
        OB_CUDA(cudaMemcpyAsync(S->b, rhs, live, cudaMemcpyDeviceToDevice, stream));
        OB_CUDA(cudaMemcpyAsync(S->x, x, live, cudaMemcpyDeviceToDevice, stream));
    } else {
        // Scatter the caller's [n][k_live] columns into the padded [n][k] layout.
        OB_CUDA(cudaMemsetAsync(S->b, 0, live, stream));
        OB_CUDA(cudaMemsetAsync(S->x, 0, live, stream));
        OB_CUDA(cudaMemcpy2DAsync(S->b, sizeof(double) * S->k, rhs, sizeof(double) * S->k_live,
                                  sizeof(double) * S->k_live, S->n, cudaMemcpyDeviceToDevice,
                                  stream));
        OB_CUDA(cudaMemcpy2DAsync(S->x, sizeof(double) * S->k, x, sizeof(double) * S->k_live,
                                  sizeof(double) * S->k_live, S->n, cudaMemcpyDeviceToDevice,
                                  stream));
    }
    OB_CUDA(cudaMemcpyAsync(S->previous, S->x, live, cudaMemcpyDeviceToDevice, stream));
    OB_CUDA(cudaMemsetAsync(S->p, 0, live, stream));
    OB_CUDA(cudaMemsetAsync(S->s, 0, live, stream));
    reset_kernel<<<S->blocks, kThreads, 0, stream>>>(S->n, S->k, S->k_live, S->b, tol, S->partials,
                                                     S->counters + 2, S->scalars, S->state,
                                                     S->settle);
    OB_CHECK_LAUNCH("reset");
    double* target = (S->precond == 1) ? S->scaled : S->u;
    initial_residual_kernel<<<S->blocks, kThreads, 0, stream>>>(
        S->n, S->k, S->offsets, S->columns, S->values, S->b, S->x, S->inv_diag, S->r, target);
    OB_CHECK_LAUNCH("initial_residual");
    if (S->precond == 1) {
        int st = enqueue_polynomial(S, stream);
        if (st) return st;
    }
    return OB_OK;
}

// Counts the kernel launches of the loop bodies the last solve replayed (read back first).
void count_body_launches(Solver* S, int rounds_per_body, int settle) {
    const int per_round = 2 + (S->precond == 1 ? kChebyshevDegree - 1 : 0);
    const long long bodies = std::max(1, (S->host_state->round + rounds_per_body - 1) / rounds_per_body);
    count_launch((uint64_t)(bodies * ((long long)rounds_per_body * per_round + settle + 1)));
}

int finish_solve(Solver* S, double* x, cudaStream_t stream) {
    const size_t live = sizeof(double) * (size_t)S->n * S->k;
    if (S->k == S->k_live)
        OB_CUDA(cudaMemcpyAsync(x, S->x, live, cudaMemcpyDeviceToDevice, stream));
    else
        OB_CUDA(cudaMemcpy2DAsync(x, sizeof(double) * S->k_live, S->x, sizeof(double) * S->k,
                                  sizeof(double) * S->k_live, S->n, cudaMemcpyDeviceToDevice,
                                  stream));
    OB_CUDA(cudaMemcpyAsync(S->host_state, S->state, sizeof(LoopState), cudaMemcpyDeviceToHost,
                            stream));
    OB_CUDA(cudaMemcpyAsync(S->host_scalars, S->scalars, sizeof(ColumnScalars) * S->k,
                            cudaMemcpyDeviceToHost, stream));
    return OB_OK;
}

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_pcg_create(int n, const int32_t* offsets, const int32_t* columns, const double* values,
                  int n_columns, int precond, int narrow, void** solver, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(solver != nullptr, "ob_pcg_create: null output");
    *solver = nullptr;
    OB_REQUIRE(n >= 1, "ob_pcg_create: n must be positive");
    OB_REQUIRE(n_columns >= 1 && n_columns <= kThreads,
               "ob_pcg_create: n_columns must be in [1, %d]", kThreads);
    OB_REQUIRE(precond == 0 || precond == 1, "ob_pcg_create: precond must be 0 or 1");
    OB_REQUIRE(offsets && columns && values, "ob_pcg_create: null CSR array");
    Solver* S = new Solver();
    S->n = n;
    S->k_live = n_columns;
    S->k = next_pow2(n_columns);
    S->precond = precond;
    S->narrow = narrow ? 1 : 0;
    int nnz = 0;
    cudaError_t e = cudaMemcpyAsync(&nnz, offsets + n, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        solver_release(S);
        return cuda_status(e, "ob_pcg_create: reading nnz");
    }
    S->nnz = nnz;
    const long long total = (long long)n * S->k;
    S->blocks = (int)std::max(1LL, std::min((total + kThreads - 1) / kThreads,
                                            (long long)8 * sm_count()));
    const size_t vec = sizeof(double) * (size_t)total;
    int st = OB_OK;
    auto A = [&](void** p, size_t bytes) {
        if (st == OB_OK) st = solver_alloc(S, p, bytes, stream);
    };
    // The solver keeps its own copy of the operator (ob_pcg_rebind copies another of the same
    // shape in): its recorded loops name these arrays.
    int *own_offsets = nullptr, *own_columns = nullptr;
    double* own_values = nullptr;
    A((void**)&own_offsets, sizeof(int) * (size_t)(n + 1));
    A((void**)&own_columns, sizeof(int) * (size_t)std::max(nnz, 1));
    A((void**)&own_values, sizeof(double) * (size_t)std::max(nnz, 1));
    A((void**)&S->inv_diag, sizeof(double) * n);
    for (double** v : {&S->b, &S->x, &S->r, &S->u, &S->w, &S->p, &S->s, &S->previous})
        A((void**)v, vec);
    if (precond == 1)
        for (double** v : {&S->scaled, &S->t0, &S->t1}) A((void**)v, vec);
    A((void**)&S->partials, sizeof(double) * 3 * (size_t)S->blocks * S->k);
    A((void**)&S->maxima, sizeof(double) * (size_t)S->blocks);
    A((void**)&S->settle_partials, sizeof(double2) * (size_t)S->blocks);
    A((void**)&S->steps, sizeof(double4) * kChebyshevDegree);
    A((void**)&S->scalars, sizeof(ColumnScalars) * S->k);
    A((void**)&S->state, sizeof(LoopState));
    A((void**)&S->settle, sizeof(SettleState));
    A((void**)&S->counters, sizeof(unsigned int) * 8);
    S->n_slices = ceil_div(n, kSlice);
    A((void**)&S->sell_start, sizeof(long long) * ((size_t)S->n_slices + 1));
    if (st != OB_OK) {
        solver_release(S);
        return st;
    }
    if (cudaMallocHost((void**)&S->host_state, sizeof(LoopState)) != cudaSuccess ||
        cudaMallocHost((void**)&S->host_scalars, sizeof(ColumnScalars) * S->k) != cudaSuccess ||
        cudaStreamCreateWithFlags(&S->capture, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        solver_release(S);
        return fail(OB_ERR_NOMEM, "ob_pcg_create: host allocations failed");
    }
    e = cudaMemsetAsync(S->counters, 0, sizeof(unsigned int) * 8, stream);
    if (e != cudaSuccess) {
        solver_release(S);
        return cuda_status(e, "ob_pcg_create: memset");
    }
    S->offsets = own_offsets;
    S->columns = own_columns;
    S->values = own_values;
    st = bind_operator(S, offsets, columns, values, stream);
    if (st == OB_OK) {
        e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) st = cuda_status(e, "ob_pcg_create: setup");
    }
    if (st != OB_OK) {
        solver_release(S);
        return st;
    }
    *solver = S;
    return OB_OK;
}

int ob_pcg_rebind(void* solver, const int32_t* offsets, const int32_t* columns, const double* values,
                  long long nnz, ob_stream_t stream_) {
    OB_REQUIRE(solver && offsets && columns && values, "ob_pcg_rebind: bad argument");
    Solver* S = static_cast<Solver*>(solver);
    OB_REQUIRE(nnz == S->nnz, "ob_pcg_rebind: %lld stored entries, the solver's shape has %lld", nnz,
               S->nnz);
    return bind_operator(S, offsets, columns, values, as_stream(stream_));
}

int ob_pcg_destroy(void* solver) {
    if (solver == nullptr) return OB_OK;
    Solver* S = static_cast<Solver*>(solver);
    {
        std::lock_guard<std::recursive_mutex> guard(capture_mutex());
        cudaDeviceSynchronize();
    }
    solver_release(S);
    return OB_OK;
}

int ob_pcg_solve(void* solver, const double* rhs, double* x, double tol, int maxiter,
                 int* iterations, double* relative_residual, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(solver && rhs && x, "ob_pcg_solve: null pointer");
    OB_REQUIRE(tol >= 0.0 && maxiter >= 0, "ob_pcg_solve: bad tolerance or cap");
    Solver* S = static_cast<Solver*>(solver);
    int st = start_solve(S, rhs, x, tol, stream);
    if (st) return st;
    st = loop_graph(S, 0, 4, maxiter, 0, 0.0, 0);
    if (st) return st;
    OB_CUDA(cudaGraphLaunch(S->exec[0], stream));
    st = finish_solve(S, x, stream);
    if (st) return st;
    if (iterations || relative_residual) {
        OB_CUDA(cudaStreamSynchronize(stream));
        count_body_launches(S, 4, 0);
        for (int c = 0; c < S->k_live; ++c) {
            if (iterations) iterations[c] = S->host_state->iterations;
            if (relative_residual) {
                const ColumnScalars& sc = S->host_scalars[c];
                relative_residual[c] = sc.rr0 > 0.0 ? sqrt(sc.rr / sc.rr0) : sqrt(sc.rr);
            }
        }
    }
    return OB_OK;
}

int ob_pcg_settle(void* solver, const double* rhs, double* x, int check_rounds,
                  double change_tolerance, int settle_rounds, int maxiter, int* rounds,
                  int* status, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(solver && rhs && x, "ob_pcg_settle: null pointer");
    OB_REQUIRE(check_rounds >= 1 && check_rounds <= 256, "ob_pcg_settle: check_rounds in [1, 256]");
    OB_REQUIRE(maxiter >= 0, "ob_pcg_settle: negative cap");
    Solver* S = static_cast<Solver*>(solver);
    int st = start_solve(S, rhs, x, 0.0, stream);
    if (st) return st;
    st = loop_graph(S, 1, check_rounds, maxiter, check_rounds, change_tolerance, settle_rounds);
    if (st) return st;
    OB_CUDA(cudaGraphLaunch(S->exec[1], stream));
    st = finish_solve(S, x, stream);
    if (st) return st;
    if (rounds || status) {
        OB_CUDA(cudaStreamSynchronize(stream));
        count_body_launches(S, check_rounds, 1);
        if (rounds) *rounds = S->host_state->iterations;
        if (status) *status = S->host_state->status;
    }
    return OB_OK;
}

int ob_pcg_time_matvec(void* solver, int reps, float* ms, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(solver && ms && reps >= 1, "ob_pcg_time_matvec: bad argument");
    Solver* S = static_cast<Solver*>(solver);
    // Each launch is timed alone, its loop state reset before it (a launch that finds the loop
    // over returns at once, and a zero residual ends the loop after one launch).
    cudaEvent_t start, end;
    OB_CUDA(cudaEventCreate(&start));
    OB_CUDA(cudaEventCreate(&end));
    int st = OB_OK;
    const int B = S->blocks;
    float total = 0.0f;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < reps && st == OB_OK && e == cudaSuccess; ++i) {
        e = cudaMemsetAsync(S->state, 0, sizeof(LoopState), stream);
        if (e != cudaSuccess) break;
        cudaEventRecord(start, stream);
        if (S->narrow)
            matvec_dots_kernel<float><<<B, kThreads, 0, stream>>>(
                S->n, S->k, sell32(S), S->r, S->u, S->w, S->partials, S->counters, S->scalars,
                S->state, 0x7fffffff);
        else
            matvec_dots_kernel<double><<<B, kThreads, 0, stream>>>(
                S->n, S->k, sell64(S), S->r, S->u, S->w, S->partials, S->counters, S->scalars,
                S->state, 0x7fffffff);
        count_launch();
        if (cudaGetLastError() != cudaSuccess) st = fail(OB_ERR_CUDA, "ob_pcg_time_matvec: launch");
        cudaEventRecord(end, stream);
        e = cudaEventSynchronize(end);
        float one = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&one, start, end);
        total += one;
    }
    cudaEventDestroy(start);
    cudaEventDestroy(end);
    if (st) return st;
    if (e != cudaSuccess) return cuda_status(e, "ob_pcg_time_matvec");
    *ms = total / (float)reps;
    // Leave the state as a finished solve would.
    OB_CUDA(cudaMemsetAsync(S->state, 0, sizeof(LoopState), stream));
    return OB_OK;
}

int ob_pcg_info(void* solver, long long* info) {
    OB_REQUIRE(solver && info, "ob_pcg_info: bad argument");
    Solver* S = static_cast<Solver*>(solver);
    info[0] = S->n;
    info[1] = S->k;
    info[2] = S->nnz;
    info[3] = S->narrow;
    info[4] = S->blocks;
    info[5] = S->sell_entries;
    return OB_OK;
}

int ob_backward_error(int n, const int32_t* offsets, const int32_t* columns, const double* values,
                      const double* x, const double* rhs, int n_columns, double tol,
                      int32_t* flag, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(flag != nullptr, "ob_backward_error: null flag");
    OB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int32_t), stream));
    if (n <= 0) return OB_OK;
    OB_REQUIRE(offsets && columns && values && x && rhs && n_columns >= 1,
               "ob_backward_error: bad argument");
    const long long total = (long long)n * n_columns;
    const int blocks = (int)std::min((total + kThreads - 1) / kThreads, (long long)8 * sm_count());
    backward_error_kernel<<<blocks, kThreads, 0, stream>>>(n, n_columns, offsets, columns, values,
                                                           x, rhs, tol, flag);
    OB_CHECK_LAUNCH("backward_error");
    return OB_OK;
}

int ob_spmv(int n, const int32_t* offsets, const int32_t* columns, const double* values,
            const double* x, double* y, int n_columns, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    if (n <= 0) return OB_OK;
    OB_REQUIRE(offsets && columns && values && x && y && n_columns >= 1, "ob_spmv: bad argument");
    const long long total = (long long)n * n_columns;
    const int blocks = (int)std::min((total + kThreads - 1) / kThreads, (long long)8 * sm_count());
    spmv_kernel<<<blocks, kThreads, 0, stream>>>(n, n_columns, offsets, columns, values, x, y);
    OB_CHECK_LAUNCH("spmv");
    return OB_OK;
}

}  // extern "C"
