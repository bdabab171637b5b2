// Smoothed-aggregation algebraic multigrid (SA-AMG) and the mixed-precision solve built on it:
// float32 preconditioned CG with a float32 V-cycle inside float64 iterative refinement.
//
// Hierarchy (host C++, once per operator) -- ordito/linalg.py:6412 (_multigrid_hierarchy) and the
// kernels of ordito/kernels/algorithms/multigrid.py it launches:
//   * strength: A_ij (j != i) is an edge when |A_ij| >= theta sqrt(|A_ii| |A_jj|), theta = 0.05
//     (multigrid.py:91, linalg.py:6340);
//   * aggregation: a distance-2 maximal independent set by randomized priorities, each round two
//     hops of a packed (state, priority, index) maximum (multigrid.py:232-361), then roots spread
//     their label two hops, largest id winning (:408); rows with no off-diagonal start excluded;
//   * smoother: l1-Jacobi, D1_ii = sign(A_ii)(|A_ii| + sum_j!=i |A_ij|), damped by
//     omega = (4/3) / rho(D1^-1 A), rho from 8 unnormalised power steps on a sign vector
//     (multigrid.py:1551-1776, linalg.py:6641);
//   * prolongator P = (I - omega D1^-1 A) P0, P0 the aggregates' normalised near-nullspace vector
//     sqrt(weights); a hub entry (a row of >= 1024 entries) does not smooth (multigrid.py:515);
//   * coarse operator P^T (A P), both products summed per output entry in the reference's slot
//     order, exact zeros pruned (linalg.py:6795, multigrid.py:649-822);
//   * coarsening stops at <= 384 rows, 12 levels, or a level that keeps >= 90 % of its rows; the
//     coarsest operator's active rows (nonzero diagonal, <= 512) get a symmetric pseudo-inverse
//     (linalg.py:7015-7125). Here the pseudo-inverse comes from a pivoted Cholesky factorisation:
//     a full-rank block is inverted through its factor, a rank-deficient one through
//     (A + N N^T)^-1 - N N^T with N an orthonormal basis of the null space the factorisation
//     exposes (the Moore-Penrose inverse of a symmetric positive semi-definite matrix).
//   The priorities and the power iteration's signs come from a SplitMix64 hash of (seed, row)
//   (Steele, Lea and Flood 2014) rather than Warp's generator, so a hierarchy is a deterministic
//   function of the operator and the seed, but not the reference's bit pattern.
//
// Cycle and solve (device). Vectors are row-interleaved float32 [n][kp] (kp a power of two >= 4
// holding the right-hand-side columns), so one row group of kp/4 lanes reads a neighbour's kp
// values as float4s -- the SpMM gather is one coalesced 16-byte load per lane. The V-cycle: the
// first pre-sweep from zero is a write (x = w D1^-1 b), one more pre-sweep, residual, restriction
// by R = P^T, the coarser cycle, prolongation added in place, two post-sweeps
// (linalg.py:7364-7434); the coarsest level multiplies by the pseudo-inverse. The solve
// (ob_amg_solve) is float64 iterative refinement: r = b - A x with the caller's float64 values,
// r scaled by its 2-norm into float32, a float32 PCG with the V-cycle to a relative inner
// tolerance, x += scale * d. Float64 is used on the device only for that residual, the
// accumulated solution and the CG dot-product reductions. The inner PCG is one CUDA graph with a
// conditional WHILE node; its body fuses q = A z + beta q with p = z + beta p (so no separate
// direction update runs) and r.z into the top level's last post-sweep.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <utility>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include "ob_host.hpp"
#include "ob_internal.cuh"
#include "ob_scratch.cuh"

namespace ob {
namespace {

constexpr double kTheta = 0.05;              // ordito/linalg.py:6340
constexpr int kMaxCoarse = 384;              // :6284
constexpr int kMaxLevels = 12;               // :6289
constexpr double kMinCoarsening = 0.9;       // :6290
constexpr int kMaxDense = 512;               // :6291
constexpr int kMaxDensified = 4096;          // :6366
constexpr int kSweeps = 2;                   // :6307
static_assert(kSweeps == 2, "enqueue_cycle is written for two sweeps a side");
constexpr double kJacobiFactor = 4.0 / 3.0;  // :6308
constexpr int kPowerSteps = 8;               // :6314
constexpr int kMisRounds = 32;               // :6315
constexpr int kLongRow = 1024;               // ordito/kernels/array.py:1197
constexpr long long kTripletFactor = 16;         // ordito/linalg.py:6347 (key budget of a product)
constexpr long long kDenseOutputCap = 1LL << 28;  // :6357 (rows x coarse columns of the fallback)

constexpr int kExcluded = 0, kUndecided = 1, kRoot = 2;  // multigrid.py:75-77

constexpr int kMaxColumns = 128;  // columns per device pass (kp <= 128: <= 32 lanes per row)
constexpr int kThreads = 256;

// ---------------------------------------------------------------------------------------------
// Host hierarchy
// ---------------------------------------------------------------------------------------------

struct HCsr {
    int rows = 0, cols = 0;
    std::vector<int> off, col;
    std::vector<double> val;
    long long nnz() const { return off.empty() ? 0 : off[rows]; }
    bool long_row(int i) const { return off[i + 1] - off[i] >= kLongRow; }
};

__host__ __device__ inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__host__ __device__ inline uint32_t row_priority(uint32_t seed, int i) {
    return (uint32_t)(splitmix64(((uint64_t)seed << 32) | (uint32_t)i) >> 36);  // 28 bits
}

__host__ __device__ inline double row_sign(uint32_t seed, int i) {
    return (splitmix64(((uint64_t)(seed ^ 0xA5A5A5A5u) << 32) | (uint32_t)i) >> 63) ? -1.0 : 1.0;
}

// The packed comparison key of multigrid.py:122: state in bits 60-61, priority 32-59, index 0-31.
__host__ __device__ inline int64_t mis_key(int state, uint32_t priority, int i) {
    return ((int64_t)state << 60) | ((int64_t)(priority & 0x0FFFFFFFu) << 32) | (int64_t)(uint32_t)i;
}

__host__ __device__ inline double inverse_or_one(double d) { return d != 0.0 ? 1.0 / d : 1.0; }

// Builds a CSR row by row: fn(i, entries) appends row i's (column, value) pairs already summed,
// sorted and pruned. Rows are produced by host threads in contiguous chunks and concatenated.
template <typename RowFn>
HCsr build_rows(int rows, int cols, bool parallel, RowFn fn) {
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const int parts = (parallel && rows >= 4096) ? (int)hw : 1;
    std::vector<std::vector<int>> counts(parts), pcol(parts);
    std::vector<std::vector<double>> pval(parts);
    auto work = [&](int p) {
        const int begin = (int)((long long)rows * p / parts), end = (int)((long long)rows * (p + 1) / parts);
        std::vector<std::pair<int, double>> entries;
        counts[p].reserve(end - begin);
        for (int i = begin; i < end; ++i) {
            entries.clear();
            fn(i, entries);
            counts[p].push_back((int)entries.size());
            for (auto& e : entries) {
                pcol[p].push_back(e.first);
                pval[p].push_back(e.second);
            }
        }
    };
    if (parts == 1) {
        work(0);
    } else {
        std::vector<std::thread> pool;
        for (int p = 1; p < parts; ++p) pool.emplace_back(work, p);
        work(0);
        for (auto& t : pool) t.join();
    }
    HCsr M;
    M.rows = rows;
    M.cols = cols;
    M.off.assign(rows + 1, 0);
    int row = 0;
    for (int p = 0; p < parts; ++p)
        for (int c : counts[p]) {
            M.off[row + 1] = M.off[row] + c;
            ++row;
        }
    M.col.reserve(M.off[rows]);
    M.val.reserve(M.off[rows]);
    for (int p = 0; p < parts; ++p) {
        M.col.insert(M.col.end(), pcol[p].begin(), pcol[p].end());
        M.val.insert(M.val.end(), pval[p].begin(), pval[p].end());
    }
    return M;
}

// Sums contributions that arrived in slot order per column (a stable sort keeps that order within
// a column), dropping exact-zero sums -- the pruned key assembly of ordito/array.py:1688.
void sum_sorted(std::vector<std::pair<int, double>>& entries) {
    std::stable_sort(entries.begin(), entries.end(),
                     [](const std::pair<int, double>& a, const std::pair<int, double>& b) {
                         return a.first < b.first;
                     });
    size_t out = 0;
    for (size_t i = 0; i < entries.size();) {
        const int c = entries[i].first;
        double s = 0.0;
        size_t j = i;
        for (; j < entries.size() && entries[j].first == c; ++j) s += entries[j].second;
        if (s != 0.0) entries[out++] = {c, s};
        i = j;
    }
    entries.resize(out);
}

HCsr transpose(const HCsr& M) {
    HCsr T;
    T.rows = M.cols;
    T.cols = M.rows;
    T.off.assign(M.cols + 1, 0);
    for (long long e = 0; e < M.nnz(); ++e) ++T.off[M.col[e] + 1];
    for (int c = 0; c < M.cols; ++c) T.off[c + 1] += T.off[c];
    T.col.resize(M.nnz());
    T.val.resize(M.nnz());
    std::vector<int> next(T.off.begin(), T.off.end() - 1);
    for (int i = 0; i < M.rows; ++i)
        for (int e = M.off[i]; e < M.off[i + 1]; ++e) {
            const int slot = next[M.col[e]]++;
            T.col[slot] = i;
            T.val[slot] = M.val[e];
        }
    return T;
}

struct Aggregation {
    std::vector<int> label;   // per row: its aggregate, -1 when unaggregated
    std::vector<int> sizes;   // per aggregate: the finest rows it stands for
    std::vector<double> l1;   // the l1 diagonal the smoother reads
    int n_aggregates = 0;
};

// ordito/linalg.py:6521 (_multigrid_aggregate) with the l1 smoother; `weights` empty on the
// finest level (every row stands for itself).
Aggregation aggregate(const HCsr& A, uint32_t seed, const std::vector<int>& weights) {
    const int n = A.rows;
    const bool par = n >= 32768;
    std::vector<double> scaled(n);
    std::vector<uint32_t> priority(n);
    std::vector<int> state(n);
    Aggregation G;
    G.l1.resize(n);
    parallel_range(n, par, [&](long long b, long long e) {
        for (int i = (int)b; i < (int)e; ++i) {
            double d = 0.0, off_sum = 0.0;
            for (int k = A.off[i]; k < A.off[i + 1]; ++k) {
                if (A.col[k] == i) d += A.val[k];
                else off_sum += std::fabs(A.val[k]);
            }
            const double l1 = std::fabs(d) + off_sum;
            G.l1[i] = d < 0.0 ? -l1 : l1;
            scaled[i] = std::sqrt(std::fabs(d));
            priority[i] = row_priority(seed, i);
            state[i] = off_sum == 0.0 ? kExcluded : kUndecided;
        }
    });
    auto strong = [&](int i, int k) {
        const int j = A.col[k];
        return j != i && std::fabs(A.val[k]) >= kTheta * scaled[i] * scaled[j];
    };
    std::vector<int64_t> key(n);
    std::vector<int> next(n);
    for (int round = 0; round < kMisRounds; ++round) {
        parallel_range(n, par, [&](long long b, long long e) {
            for (int i = (int)b; i < (int)e; ++i) {
                int64_t best = mis_key(state[i], priority[i], i);
                for (int k = A.off[i]; k < A.off[i + 1]; ++k)
                    if (strong(i, k)) {
                        const int j = A.col[k];
                        best = std::max(best, mis_key(state[j], priority[j], j));
                    }
                key[i] = best;
            }
        });
        std::atomic<long long> undecided_total(0);
        parallel_range(n, par, [&](long long b, long long e) {
            long long undecided = 0;
            for (int i = (int)b; i < (int)e; ++i) {
                if (state[i] != kUndecided) {
                    next[i] = state[i];
                    continue;
                }
                int64_t best = key[i];
                for (int k = A.off[i]; k < A.off[i + 1]; ++k)
                    if (strong(i, k)) best = std::max(best, key[A.col[k]]);
                int verdict = kUndecided;
                if ((int)(best >> 60) == kRoot) verdict = kExcluded;
                else if (best == mis_key(kUndecided, priority[i], i)) verdict = kRoot;
                next[i] = verdict;
                undecided += verdict == kUndecided;
            }
            undecided_total += undecided;
        });
        state.swap(next);
        if (undecided_total.load() == 0) break;
    }
    // Aggregates: every node not excluded (roots, and any left undecided by the round cap).
    std::vector<int> label0(n, -1);
    int count = 0;
    for (int i = 0; i < n; ++i)
        if (state[i] != kExcluded) label0[i] = count++;
    G.n_aggregates = count;
    // Two hops of the spread over the strong graph, largest label winning.
    std::vector<int> hop(n);
    parallel_range(n, par, [&](long long b, long long e) {
        for (int i = (int)b; i < (int)e; ++i) {
            int best = label0[i];
            if (best < 0)
                for (int k = A.off[i]; k < A.off[i + 1]; ++k)
                    if (strong(i, k)) best = std::max(best, label0[A.col[k]]);
            hop[i] = best;
        }
    });
    G.label.assign(n, -1);
    parallel_range(n, par, [&](long long b, long long e) {
        for (int i = (int)b; i < (int)e; ++i) {
            int best = hop[i];
            if (best < 0)
                for (int k = A.off[i]; k < A.off[i + 1]; ++k)
                    if (strong(i, k)) best = std::max(best, hop[A.col[k]]);
            G.label[i] = best;
        }
    });
    G.sizes.assign(count, 0);
    for (int i = 0; i < n; ++i)
        if (G.label[i] >= 0) G.sizes[G.label[i]] += weights.empty() ? 1 : weights[i];
    return G;
}

// omega D1^-1 with omega = (4/3) / rho(D1^-1 A), rho from the growth of 8 unnormalised power steps
// on a sign vector (ordito/linalg.py:6641, multigrid.py:1551).
std::vector<double> damped_diagonal(const HCsr& A, const std::vector<double>& l1, uint32_t seed) {
    const int n = A.rows;
    const bool par = n >= 32768;
    std::vector<double> x(n), y(n);
    for (int i = 0; i < n; ++i) x[i] = row_sign(seed, i);
    for (int step = 0; step < kPowerSteps; ++step) {
        parallel_range(n, par, [&](long long b, long long e) {
            for (int i = (int)b; i < (int)e; ++i) {
                double t = 0.0;
                for (int k = A.off[i]; k < A.off[i + 1]; ++k) t += A.val[k] * x[A.col[k]];
                y[i] = inverse_or_one(l1[i]) * t;
            }
        });
        x.swap(y);
    }
    double growth = 0.0;
    for (int i = 0; i < n; ++i) growth += x[i] * x[i];
    double rho = 1.0;
    if (n > 0 && growth > 0.0 && std::isfinite(growth))
        rho = std::pow(std::sqrt(growth / (double)n), 1.0 / kPowerSteps);
    const double omega = kJacobiFactor / rho;
    std::vector<double> damped(n);
    for (int i = 0; i < n; ++i) damped[i] = omega * inverse_or_one(l1[i]);
    return damped;
}

// P = (I - omega D1^-1 A) P0 (multigrid.py:515-630).
HCsr prolongator(const HCsr& A, const Aggregation& G, const std::vector<int>& weights,
                 const std::vector<double>& damped) {
    const int n = A.rows;
    auto scale_of = [&](int i) { return weights.empty() ? 1.0 : std::sqrt((double)weights[i]); };
    auto norm_of = [&](int a) { return std::sqrt((double)G.sizes[a]); };
    return build_rows(n, G.n_aggregates, n >= 32768, [&](int i, std::vector<std::pair<int, double>>& out) {
        const double scale = -damped[i];
        for (int k = A.off[i]; k < A.off[i + 1]; ++k) {
            const int j = A.col[k];
            const int a = G.label[j];
            const bool hub = j != i && (A.long_row(i) || A.long_row(j));
            if (a < 0 || hub) continue;
            const double c = scale * A.val[k] * scale_of(j) / norm_of(a);
            if (c != 0.0) out.push_back({a, c});
        }
        const int own = G.label[i];
        if (own >= 0) {
            const double c = scale_of(i) / norm_of(own);
            if (c != 0.0) out.push_back({own, c});
        }
        sum_sorted(out);
    });
}

// A P then P^T (A P), each entry summed in the reference's contribution order. Row by row, so
// memory follows the products' output and one path serves both of the reference's (its key
// assembly and, past the key budget, bsr_mm: ordito/linalg.py:6842-6898). False -- the hierarchy
// ends at this level -- where the reference ends it: a product past its key budget whose
// rows x coarse columns is also past the fallback's cap.
bool galerkin(const HCsr& A, const HCsr& P, const HCsr& R, HCsr* out) {
    const long long budget = kTripletFactor * (A.nnz() + A.rows);
    const bool capped = (long long)A.rows * P.cols > kDenseOutputCap;
    long long contributions = 0;
    for (int i = 0; i < A.rows; ++i)
        for (int k = A.off[i]; k < A.off[i + 1]; ++k) {
            const int j = A.col[k];
            contributions += P.off[j + 1] - P.off[j];
        }
    if (contributions > budget && capped) return false;
    HCsr AP = build_rows(A.rows, P.cols, A.rows >= 32768, [&](int i, std::vector<std::pair<int, double>>& o) {
        for (int k = A.off[i]; k < A.off[i + 1]; ++k) {
            const int j = A.col[k];
            const double a = A.val[k];
            for (int b = P.off[j]; b < P.off[j + 1]; ++b) {
                const double c = a * P.val[b];
                if (c != 0.0) o.push_back({P.col[b], c});
            }
        }
        sum_sorted(o);
    });
    contributions = 0;
    for (int c = 0; c < R.rows; ++c)
        for (int k = R.off[c]; k < R.off[c + 1]; ++k) {
            const int i = R.col[k];
            contributions += AP.off[i + 1] - AP.off[i];
        }
    if (contributions > budget && capped) return false;
    *out = build_rows(R.rows, P.cols, R.rows >= 32768, [&](int c, std::vector<std::pair<int, double>>& o) {
        for (int k = R.off[c]; k < R.off[c + 1]; ++k) {
            const int i = R.col[k];
            const double p = R.val[k];
            for (int b = AP.off[i]; b < AP.off[i + 1]; ++b) {
                const double v = p * AP.val[b];
                if (v != 0.0) o.push_back({AP.col[b], v});
            }
        }
        sum_sorted(o);
    });
    return true;
}

// Symmetric pseudo-inverse of the dense symmetric positive semi-definite m x m matrix S
// (row-major) by pivoted Cholesky: full rank -> S^-1 from the factor; rank r < m -> with N an
// orthonormal basis of the null space the factor exposes, (S + N N^T)^-1 - N N^T. Returns false
// when S is not positive semi-definite to rounding.
bool cholesky_inverse(std::vector<double>& a, int m) {
    // In-place lower Cholesky of a (row-major, lower part) then the inverse of L^T L... a = S.
    for (int j = 0; j < m; ++j) {
        double d = a[(size_t)j * m + j];
        for (int k = 0; k < j; ++k) d -= a[(size_t)j * m + k] * a[(size_t)j * m + k];
        if (!(d > 0.0)) return false;
        d = std::sqrt(d);
        a[(size_t)j * m + j] = d;
        for (int i = j + 1; i < m; ++i) {
            double s = a[(size_t)i * m + j];
            for (int k = 0; k < j; ++k) s -= a[(size_t)i * m + k] * a[(size_t)j * m + k];
            a[(size_t)i * m + j] = s / d;
        }
    }
    // W = L^-1 (lower), row-major in w.
    std::vector<double> w((size_t)m * m, 0.0);
    for (int c = 0; c < m; ++c) {
        w[(size_t)c * m + c] = 1.0 / a[(size_t)c * m + c];
        for (int i = c + 1; i < m; ++i) {
            double s = 0.0;
            for (int k = c; k < i; ++k) s -= a[(size_t)i * m + k] * w[(size_t)k * m + c];
            w[(size_t)i * m + c] = s / a[(size_t)i * m + i];
        }
    }
    // S^-1 = W^T W.
    for (int i = 0; i < m; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
            for (int k = i; k < m; ++k) s += w[(size_t)k * m + i] * w[(size_t)k * m + j];
            a[(size_t)i * m + j] = s;
            a[(size_t)j * m + i] = s;
        }
    return true;
}

bool symmetric_pseudo_inverse(const std::vector<double>& S, int m, std::vector<double>* out) {
    std::vector<double> a(S);
    std::vector<int> piv(m);
    for (int i = 0; i < m; ++i) piv[i] = i;
    double max_diag = 0.0;
    for (int i = 0; i < m; ++i) max_diag = std::max(max_diag, std::fabs(S[(size_t)i * m + i]));
    const double tol = std::max(1e-300, 1e-12 * max_diag * m);
    // Pivoted outer-product Cholesky on a permuted copy b (row-major full symmetric).
    std::vector<double> b(S);
    int rank = 0;
    for (; rank < m; ++rank) {
        int best = rank;
        for (int i = rank + 1; i < m; ++i)
            if (b[(size_t)i * m + i] > b[(size_t)best * m + best]) best = i;
        if (!(b[(size_t)best * m + best] > tol)) break;
        if (best != rank) {
            std::swap(piv[rank], piv[best]);
            for (int k = 0; k < m; ++k) std::swap(b[(size_t)rank * m + k], b[(size_t)best * m + k]);
            for (int k = 0; k < m; ++k) std::swap(b[(size_t)k * m + rank], b[(size_t)k * m + best]);
        }
        const double d = std::sqrt(b[(size_t)rank * m + rank]);
        b[(size_t)rank * m + rank] = d;
        for (int i = rank + 1; i < m; ++i) b[(size_t)i * m + rank] /= d;
        for (int j = rank + 1; j < m; ++j) {
            const double lj = b[(size_t)j * m + rank];
            for (int i = j; i < m; ++i) {
                b[(size_t)i * m + j] -= b[(size_t)i * m + rank] * lj;
                b[(size_t)j * m + i] = b[(size_t)i * m + j];
            }
        }
    }
    const int null_dim = m - rank;
    std::vector<double> N((size_t)m * std::max(null_dim, 1), 0.0);  // column-major m x null_dim
    if (null_dim > 0) {
        // Null vectors in pivoted order: [-L11^-T L21^T; I], L11 = b[0:r, 0:r], L21 = b[r:, 0:r].
        for (int t = 0; t < null_dim; ++t) {
            std::vector<double> v(m, 0.0);
            v[rank + t] = 1.0;
            // Solve L11^T y = -L21[t, :]^T (back substitution).
            for (int i = rank - 1; i >= 0; --i) {
                double s = -b[(size_t)(rank + t) * m + i];
                for (int k = i + 1; k < rank; ++k) s -= b[(size_t)k * m + i] * v[k];
                v[i] = s / b[(size_t)i * m + i];
            }
            double* col = N.data() + (size_t)t * m;
            for (int i = 0; i < m; ++i) col[piv[i]] = v[i];
        }
        // Orthonormalise (modified Gram-Schmidt, twice).
        for (int pass = 0; pass < 2; ++pass)
            for (int t = 0; t < null_dim; ++t) {
                double* col = N.data() + (size_t)t * m;
                for (int u = 0; u < t; ++u) {
                    const double* prev = N.data() + (size_t)u * m;
                    double dot = 0.0;
                    for (int i = 0; i < m; ++i) dot += prev[i] * col[i];
                    for (int i = 0; i < m; ++i) col[i] -= dot * prev[i];
                }
                double norm = 0.0;
                for (int i = 0; i < m; ++i) norm += col[i] * col[i];
                norm = std::sqrt(norm);
                if (!(norm > 0.0)) return false;
                for (int i = 0; i < m; ++i) col[i] /= norm;
            }
        // Shift the null space onto a scale comparable to the rest of the spectrum.
        for (int t = 0; t < null_dim; ++t) {
            const double* col = N.data() + (size_t)t * m;
            for (int i = 0; i < m; ++i)
                for (int j = 0; j < m; ++j) a[(size_t)i * m + j] += max_diag * col[i] * col[j];
        }
    }
    if (!cholesky_inverse(a, m)) return false;
    if (null_dim > 0)
        for (int t = 0; t < null_dim; ++t) {
            const double* col = N.data() + (size_t)t * m;
            for (int i = 0; i < m; ++i)
                for (int j = 0; j < m; ++j) a[(size_t)i * m + j] -= col[i] * col[j] / max_diag;
        }
    out->assign((size_t)m * m, 0.0);
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j)
            (*out)[(size_t)i * m + j] = 0.5 * (a[(size_t)i * m + j] + a[(size_t)j * m + i]);
    return true;
}

struct HostLevel {
    HCsr A;                      // this level's operator
    std::vector<double> damped;  // omega D1^-1 (empty on the coarsest level)
    HCsr P, R;                   // prolongator to this level from the next, and its transpose
};

struct HostHierarchy {
    std::vector<HostLevel> levels;  // the last is the coarsest
    std::vector<int> active;        // coarsest level's active rows (nonzero diagonal)
    std::vector<double> inverse;    // their pseudo-inverse (active x active, row-major)
    std::vector<double> jacobi;     // inverse_or_one of the fine diagonal (the no-hierarchy case)
    bool usable = false;
};

void finish_hierarchy(HostHierarchy* H);

// The hierarchy from level `first_level` on (levels before it were built elsewhere: on the
// device), A that level's operator and `weights` its rows' aggregate sizes (empty on the finest
// level); may_coarsen = false keeps A as the coarsest level.
void build_hierarchy_from(HCsr A, uint32_t seed, std::vector<int> weights, int first_level, bool may_coarsen,
                          HostHierarchy* H) {
    while (true) {
        H->levels.emplace_back();
        HostLevel& level = H->levels.back();
        if (!may_coarsen || A.rows <= kMaxCoarse || first_level + (int)H->levels.size() >= kMaxLevels) {
            level.A = std::move(A);
            break;
        }
        Aggregation G = aggregate(A, seed, weights);
        if (G.n_aggregates == 0 || G.n_aggregates >= kMinCoarsening * A.rows) {
            level.A = std::move(A);
            break;
        }
        std::vector<double> damped = damped_diagonal(A, G.l1, seed);
        HCsr P = prolongator(A, G, weights, damped);
        HCsr R = transpose(P);
        HCsr coarse;
        if (!galerkin(A, P, R, &coarse)) {
            level.A = std::move(A);
            break;
        }
        level.A = std::move(A);
        level.damped = std::move(damped);
        level.P = std::move(P);
        level.R = std::move(R);
        weights = std::move(G.sizes);
        A = std::move(coarse);
    }
    finish_hierarchy(H);
}

void build_hierarchy(HCsr fine, uint32_t seed, HostHierarchy* H) {
    H->jacobi.resize(fine.rows);
    for (int i = 0; i < fine.rows; ++i) {
        double d = 0.0;
        for (int k = fine.off[i]; k < fine.off[i + 1]; ++k)
            if (fine.col[k] == i) d += fine.val[k];
        H->jacobi[i] = inverse_or_one(d);
    }
    build_hierarchy_from(std::move(fine), seed, {}, 0, true, H);
}

// The coarsest level's dense pseudo-inverse over its active rows (the hierarchy is usable only
// with it).
void finish_hierarchy(HostHierarchy* H) {
    const HCsr& last = H->levels.back().A;
    // A single level (an operator of <= 384 rows, or one whose first aggregation stalls) is solved
    // by its dense pseudo-inverse alone, as the reference's one-level cycle is.
    if (last.rows > kMaxDensified) return;
    std::vector<int> active;
    std::vector<double> diag(last.rows, 0.0);
    for (int i = 0; i < last.rows; ++i)
        for (int k = last.off[i]; k < last.off[i + 1]; ++k)
            if (last.col[k] == i) diag[i] += last.val[k];
    for (int i = 0; i < last.rows; ++i)
        if (diag[i] != 0.0) active.push_back(i);
    if ((int)active.size() > kMaxDense) return;
    const int m = (int)active.size();
    std::vector<int> slot(last.rows, -1);
    for (int t = 0; t < m; ++t) slot[active[t]] = t;
    std::vector<double> dense((size_t)std::max(m, 1) * std::max(m, 1), 0.0);
    for (int i = 0; i < last.rows; ++i)
        for (int k = last.off[i]; k < last.off[i + 1]; ++k)
            if (slot[i] >= 0 && slot[last.col[k]] >= 0)
                dense[(size_t)slot[i] * m + slot[last.col[k]]] += last.val[k];
    if (m > 0 && !symmetric_pseudo_inverse(dense, m, &H->inverse)) return;
    H->active = std::move(active);
    H->usable = true;
}

// ---------------------------------------------------------------------------------------------
// Device hierarchy: the levels of at least kDeviceLevelRows rows are built on the device, with the
// host's arithmetic in the host's order (the same aggregates, prolongators and Galerkin operators
// as build_hierarchy for the same seed); the smaller levels and the coarse pseudo-inverse follow
// on the host from where the device stopped.
// ---------------------------------------------------------------------------------------------

constexpr int kDeviceLevelRows = 32768;

struct DevCsr {
    int rows = 0, cols = 0;
    long long nnz = 0;
    const int* off = nullptr;
    const int* col = nullptr;
    const double* val = nullptr;
};

struct DevLevel {
    DevCsr A, P, R;               // P, R empty on the last level
    const double* damped = nullptr;
};

struct DevBuild {
    std::vector<DevLevel> levels;  // the last one is where the host takes over (its A only)
    std::vector<int> weights;      // the last level's row weights (empty: the finest level)
    bool stopped = false;          // the device loop itself ended the hierarchy at the last level
    std::vector<void*> owned;      // pool allocations of the kept arrays
};

template <typename T>
int keep_alloc(DevBuild* B, T** p, size_t n, cudaStream_t stream) {
    void* q = nullptr;
    OB_CUDA(pool_malloc(&q, sizeof(T) * std::max<size_t>(n, 1), stream));
    B->owned.push_back(q);
    *p = static_cast<T*>(q);
    return OB_OK;
}

__device__ __forceinline__ bool strong_edge(int i, int j, double a, const double* __restrict__ scaled) {
    return j != i && fabs(a) >= kTheta * scaled[i] * scaled[j];
}

__global__ void dev_setup_kernel(int n, const int* __restrict__ off, const int* __restrict__ col,
                                 const double* __restrict__ val, uint32_t seed, double* __restrict__ l1,
                                 double* __restrict__ scaled, uint32_t* __restrict__ priority, int* __restrict__ state) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 0.0, off_sum = 0.0;
    for (int k = off[i]; k < off[i + 1]; ++k) {
        if (col[k] == i) d += val[k];
        else off_sum += fabs(val[k]);
    }
    const double l = fabs(d) + off_sum;
    l1[i] = d < 0.0 ? -l : l;
    scaled[i] = sqrt(fabs(d));
    priority[i] = row_priority(seed, i);
    state[i] = off_sum == 0.0 ? kExcluded : kUndecided;
}

__global__ void dev_mis_keys_kernel(int n, const int* __restrict__ off, const int* __restrict__ col,
                                    const double* __restrict__ val, const double* __restrict__ scaled,
                                    const int* __restrict__ state, const uint32_t* __restrict__ priority,
                                    int64_t* __restrict__ key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t best = mis_key(state[i], priority[i], i);
    for (int k = off[i]; k < off[i + 1]; ++k) {
        const int j = col[k];
        if (strong_edge(i, j, val[k], scaled)) best = max(best, mis_key(state[j], priority[j], j));
    }
    key[i] = best;
}

__global__ void dev_mis_decide_kernel(int n, const int* __restrict__ off, const int* __restrict__ col,
                                      const double* __restrict__ val, const double* __restrict__ scaled,
                                      const int* __restrict__ state, const uint32_t* __restrict__ priority,
                                      const int64_t* __restrict__ key, int* __restrict__ next, int* undecided) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (state[i] != kUndecided) {
        next[i] = state[i];
        return;
    }
    int64_t best = key[i];
    for (int k = off[i]; k < off[i + 1]; ++k) {
        const int j = col[k];
        if (strong_edge(i, j, val[k], scaled)) best = max(best, key[j]);
    }
    int verdict = kUndecided;
    if ((int)(best >> 60) == kRoot) verdict = kExcluded;
    else if (best == mis_key(kUndecided, priority[i], i)) verdict = kRoot;
    next[i] = verdict;
    if (verdict == kUndecided) atomicAdd(undecided, 1);
}

__global__ void dev_root_flags_kernel(int n, const int* __restrict__ state, int* __restrict__ flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flags[i] = state[i] != kExcluded ? 1 : 0;
}

__global__ void dev_first_labels_kernel(int n, const int* __restrict__ flags, const int* __restrict__ scan,
                                        int* __restrict__ label) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) label[i] = flags[i] ? scan[i] : -1;
}

// One hop of the label spread over the strong graph, the largest label winning.
__global__ void dev_spread_kernel(int n, const int* __restrict__ off, const int* __restrict__ col,
                                  const double* __restrict__ val, const double* __restrict__ scaled,
                                  const int* __restrict__ in, int* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int best = in[i];
    if (best < 0)
        for (int k = off[i]; k < off[i + 1]; ++k)
            if (strong_edge(i, col[k], val[k], scaled)) best = max(best, in[col[k]]);
    out[i] = best;
}

__global__ void dev_sizes_kernel(int n, const int* __restrict__ label, const int* __restrict__ weights,
                                 int* __restrict__ sizes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && label[i] >= 0) atomicAdd(&sizes[label[i]], weights ? weights[i] : 1);
}

__global__ void dev_signs_kernel(int n, uint32_t seed, double* __restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = row_sign(seed, i);
}

__global__ void dev_power_kernel(int n, const int* __restrict__ off, const int* __restrict__ col,
                                 const double* __restrict__ val, const double* __restrict__ l1,
                                 const double* __restrict__ x, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double t = 0.0;
    for (int k = off[i]; k < off[i + 1]; ++k) t += val[k] * x[col[k]];
    y[i] = inverse_or_one(l1[i]) * t;
}

__global__ void dev_damped_kernel(int n, const double* __restrict__ l1, double omega, double* __restrict__ damped) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) damped[i] = omega * inverse_or_one(l1[i]);
}

// Rows assembled from (column, value) contributions in slot order: FILL == false counts each row's
// non-zero contributions (and, in raw, every contribution, for the key budget); FILL == true writes
// them from the row's start as keys row * cols + col and values.

// The prolongator's contributions (prolongator(): A's entries, then the row's own aggregate).
template <bool FILL>
__global__ void dev_prolongator_kernel(int n, int n_coarse, const int* __restrict__ off, const int* __restrict__ col,
                                       const double* __restrict__ val, const int* __restrict__ label,
                                       const int* __restrict__ weights, const int* __restrict__ sizes,
                                       const double* __restrict__ damped, long long* __restrict__ count,
                                       const long long* __restrict__ start, unsigned long long* __restrict__ keys,
                                       double* __restrict__ values) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double scale = -damped[i];
    const bool long_i = off[i + 1] - off[i] >= kLongRow;
    long long c = 0, e = FILL ? start[i] : 0;
    auto emit = [&](int a, double v) {
        if (v == 0.0) return;
        if (FILL) {
            keys[e] = (unsigned long long)i * (unsigned long long)n_coarse + (unsigned long long)a;
            values[e] = v;
            ++e;
        }
        ++c;
    };
    for (int k = off[i]; k < off[i + 1]; ++k) {
        const int j = col[k];
        const int a = label[j];
        const bool hub = j != i && (long_i || off[j + 1] - off[j] >= kLongRow);
        if (a < 0 || hub) continue;
        const double scale_j = weights ? sqrt((double)weights[j]) : 1.0;
        emit(a, scale * val[k] * scale_j / sqrt((double)sizes[a]));
    }
    const int own = label[i];
    if (own >= 0) emit(own, (weights ? sqrt((double)weights[i]) : 1.0) / sqrt((double)sizes[own]));
    if (!FILL) count[i] = c;
}

// A B's contributions (galerkin()'s A P and R (A P)): row i, for each of its entries (j, a) in
// order, B's row j in order, a * b.
template <bool FILL>
__global__ void dev_product_kernel(int n, int cols, const int* __restrict__ aoff, const int* __restrict__ acol,
                                   const double* __restrict__ aval, const int* __restrict__ boff,
                                   const int* __restrict__ bcol, const double* __restrict__ bval,
                                   long long* __restrict__ count, long long* __restrict__ raw,
                                   const long long* __restrict__ start, unsigned long long* __restrict__ keys,
                                   double* __restrict__ values) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    long long c = 0, all = 0, e = FILL ? start[i] : 0;
    for (int k = aoff[i]; k < aoff[i + 1]; ++k) {
        const int j = acol[k];
        const double a = aval[k];
        all += boff[j + 1] - boff[j];
        for (int b = boff[j]; b < boff[j + 1]; ++b) {
            const double v = a * bval[b];
            if (v == 0.0) continue;
            if (FILL) {
                keys[e] = (unsigned long long)i * (unsigned long long)cols + (unsigned long long)bcol[b];
                values[e] = v;
                ++e;
            }
            ++c;
        }
    }
    if (!FILL) {
        count[i] = c;
        raw[i] = all;
    }
}

__global__ void dev_run_flags_kernel(long long total, const unsigned long long* __restrict__ keys, int* __restrict__ flags) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e < total) flags[e] = (e == 0 || keys[e] != keys[e - 1]) ? 1 : 0;
}

__global__ void dev_run_starts_kernel(long long total, const int* __restrict__ flags, const int* __restrict__ run,
                                      long long* __restrict__ first) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e < total && flags[e]) first[run[e]] = e;
}

// Each run (one output entry): its contributions summed in sorted order (slot order: the sort is
// stable), kept when the sum is not zero (sum_sorted()).
__global__ void dev_run_sums_kernel(int runs, long long total, const long long* __restrict__ first,
                                    const unsigned long long* __restrict__ keys, const int* __restrict__ perm,
                                    const double* __restrict__ values, int cols, double* __restrict__ sum,
                                    int* __restrict__ keep, int* __restrict__ row_count) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= runs) return;
    const long long b = first[r], e = r + 1 < runs ? first[r + 1] : total;
    double s = 0.0;
    for (long long t = b; t < e; ++t) s += values[perm[t]];
    sum[r] = s;
    keep[r] = s != 0.0 ? 1 : 0;
    if (s != 0.0) atomicAdd(&row_count[(int)(keys[b] / (unsigned long long)cols)], 1);
}

__global__ void dev_place_kernel(int runs, const long long* __restrict__ first, const unsigned long long* __restrict__ keys,
                                 const double* __restrict__ sum, const int* __restrict__ keep,
                                 const int* __restrict__ pos, int cols, int* __restrict__ col, double* __restrict__ val) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= runs || !keep[r]) return;
    col[pos[r]] = (int)(keys[first[r]] % (unsigned long long)cols);
    val[pos[r]] = sum[r];
}

__global__ void dev_entry_rows_kernel(int rows, const int* __restrict__ off, int* __restrict__ row) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    for (int k = off[i]; k < off[i + 1]; ++k) row[k] = i;
}

__global__ void dev_transpose_keys_kernel(long long nnz, const int* __restrict__ col, const int* __restrict__ row,
                                          int rows, unsigned long long* __restrict__ keys, int* __restrict__ index,
                                          int* __restrict__ count) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    keys[e] = (unsigned long long)col[e] * (unsigned long long)rows + (unsigned long long)row[e];
    index[e] = (int)e;
    atomicAdd(&count[col[e]], 1);
}

__global__ void dev_transpose_place_kernel(long long nnz, const unsigned long long* __restrict__ keys,
                                           const int* __restrict__ index, const double* __restrict__ val, int rows,
                                           int* __restrict__ tcol, double* __restrict__ tval) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    tcol[e] = (int)(keys[e] % (unsigned long long)rows);
    tval[e] = val[index[e]];
}

__global__ void dev_iota_kernel(long long total, int* __restrict__ index) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e < total) index[e] = (int)e;
}

int bits_for(unsigned long long value) {
    int bits = 1;
    while (bits < 64 && (value >> bits) != 0) ++bits;
    return bits;
}

int grid_of(long long n) { return (int)std::max(1LL, (n + kThreads - 1) / kThreads); }

// Exclusive scan of n ints (or long longs) into out (n + 1 entries, the total last).
template <typename T>
int exclusive_scan(const T* in, T* out, int n, cudaStream_t stream) {
    Scratch scratch(stream);
    size_t bytes = 0;
    OB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n + 1, stream));
    void* temp = scratch.take<unsigned char>(bytes);
    if (int st = scratch.commit()) return st;
    // The scan covers n + 1 entries: the input's entry n must be 0 (callers allocate n + 1 zeroed
    // at the end).
    OB_CUDA(cub::DeviceScan::ExclusiveSum(temp, bytes, in, out, n + 1, stream));
    return OB_OK;
}

template <typename T>
T read_one(const T* p, cudaStream_t stream, int* status) {
    T v{};
    cudaError_t e = cudaMemcpyAsync(&v, p, sizeof(T), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) *status = cuda_status(e, "amg device build: read back");
    return v;
}

// CSR rows x cols from per-row contributions: count (rows + 1, the last 0) is filled by the
// counting pass; fill(start, keys, values) writes them. Contributions of one entry are summed in
// their slot order (a stable radix sort over the key bits), exact-zero sums are dropped.
template <typename Fill>
int assemble(int rows, int cols, long long* count, Fill fill, DevBuild* B, DevCsr* out, cudaStream_t stream) {
    int st = OB_OK;
    Scratch scratch(stream);
    long long* start = scratch.take<long long>((size_t)rows + 1);
    if ((st = scratch.commit())) return st;
    if ((st = exclusive_scan(count, start, rows, stream))) return st;
    const long long total = read_one(start + rows, stream, &st);
    if (st) return st;
    OB_REQUIRE(total < (1LL << 31), "amg device build: %lld contributions past the index range", total);
    int* row_off = nullptr;
    if ((st = keep_alloc(B, &row_off, (size_t)rows + 1, stream))) return st;
    int* col = nullptr;
    double* val = nullptr;
    if (total == 0) {
        OB_CUDA(cudaMemsetAsync(row_off, 0, sizeof(int) * ((size_t)rows + 1), stream));
        if ((st = keep_alloc(B, &col, 1, stream)) || (st = keep_alloc(B, &val, 1, stream))) return st;
        *out = DevCsr{rows, cols, 0, row_off, col, val};
        return OB_OK;
    }
    unsigned long long* keys = scratch.take<unsigned long long>((size_t)total);
    unsigned long long* sorted = scratch.take<unsigned long long>((size_t)total);
    double* values = scratch.take<double>((size_t)total);
    int* index = scratch.take<int>((size_t)total);
    int* perm = scratch.take<int>((size_t)total);
    int* flags = scratch.take<int>((size_t)total + 1);
    int* run = scratch.take<int>((size_t)total + 1);
    if ((st = scratch.commit())) return st;
    fill(start, keys, values);
    OB_CHECK_LAUNCH("amg device build: contributions");
    dev_iota_kernel<<<grid_of(total), kThreads, 0, stream>>>(total, index);
    OB_CHECK_LAUNCH("amg device build: positions");
    OB_CUDA(cudaMemsetAsync(flags + total, 0, sizeof(int), stream));
    {
        Scratch sort_scratch(stream);
        size_t bytes = 0;
        const int end_bit = bits_for((unsigned long long)rows * (unsigned long long)cols);
        OB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, sorted, index, perm, (int)total, 0, end_bit,
                                                stream));
        void* temp = sort_scratch.take<unsigned char>(bytes);
        if ((st = sort_scratch.commit())) return st;
        OB_CUDA(cub::DeviceRadixSort::SortPairs(temp, bytes, keys, sorted, index, perm, (int)total, 0, end_bit,
                                                stream));
    }
    dev_run_flags_kernel<<<grid_of(total), kThreads, 0, stream>>>(total, sorted, flags);
    OB_CHECK_LAUNCH("amg device build: run flags");
    if ((st = exclusive_scan(flags, run, (int)total, stream))) return st;
    const int runs = read_one(run + total, stream, &st);
    if (st) return st;
    long long* first = scratch.take<long long>((size_t)runs + 1);
    double* sum = scratch.take<double>((size_t)runs + 1);
    int* keep = scratch.take<int>((size_t)runs + 1);
    int* pos = scratch.take<int>((size_t)runs + 1);
    int* row_count = scratch.take<int>((size_t)rows + 1);
    if ((st = scratch.commit())) return st;
    dev_run_starts_kernel<<<grid_of(total), kThreads, 0, stream>>>(total, flags, run, first);
    OB_CHECK_LAUNCH("amg device build: run starts");
    OB_CUDA(cudaMemsetAsync(row_count, 0, sizeof(int) * ((size_t)rows + 1), stream));
    OB_CUDA(cudaMemsetAsync(keep + runs, 0, sizeof(int), stream));
    dev_run_sums_kernel<<<grid_of(runs), kThreads, 0, stream>>>(runs, total, first, sorted, perm, values, cols, sum,
                                                                keep, row_count);
    OB_CHECK_LAUNCH("amg device build: run sums");
    if ((st = exclusive_scan(row_count, row_off, rows, stream))) return st;
    if ((st = exclusive_scan(keep, pos, runs, stream))) return st;
    const int kept = read_one(pos + runs, stream, &st);
    if (st) return st;
    if ((st = keep_alloc(B, &col, (size_t)kept, stream)) || (st = keep_alloc(B, &val, (size_t)kept, stream))) return st;
    dev_place_kernel<<<grid_of(runs), kThreads, 0, stream>>>(runs, first, sorted, sum, keep, pos, cols, col, val);
    OB_CHECK_LAUNCH("amg device build: place");
    *out = DevCsr{rows, cols, kept, row_off, col, val};
    return OB_OK;
}

// The transpose of a device CSR (rows x cols) in row order within each column (transpose()).
int transpose_device(const DevCsr& M, DevBuild* B, DevCsr* out, cudaStream_t stream) {
    int st = OB_OK;
    Scratch scratch(stream);
    const long long nnz = M.nnz;
    int* row = scratch.take<int>((size_t)std::max(nnz, 1LL));
    unsigned long long* keys = scratch.take<unsigned long long>((size_t)std::max(nnz, 1LL));
    unsigned long long* sorted = scratch.take<unsigned long long>((size_t)std::max(nnz, 1LL));
    int* index = scratch.take<int>((size_t)std::max(nnz, 1LL));
    int* perm = scratch.take<int>((size_t)std::max(nnz, 1LL));
    int* count = scratch.take<int>((size_t)M.cols + 1);
    if ((st = scratch.commit())) return st;
    int *off = nullptr, *col = nullptr;
    double* val = nullptr;
    if ((st = keep_alloc(B, &off, (size_t)M.cols + 1, stream)) || (st = keep_alloc(B, &col, (size_t)nnz, stream)) ||
        (st = keep_alloc(B, &val, (size_t)nnz, stream)))
        return st;
    OB_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * ((size_t)M.cols + 1), stream));
    if (nnz > 0) {
        dev_entry_rows_kernel<<<grid_of(M.rows), kThreads, 0, stream>>>(M.rows, M.off, row);
        OB_CHECK_LAUNCH("amg device build: entry rows");
        dev_transpose_keys_kernel<<<grid_of(nnz), kThreads, 0, stream>>>(nnz, M.col, row, M.rows, keys, index, count);
        OB_CHECK_LAUNCH("amg device build: transpose keys");
        Scratch sort_scratch(stream);
        size_t bytes = 0;
        const int end_bit = bits_for((unsigned long long)M.cols * (unsigned long long)M.rows);
        OB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, sorted, index, perm, (int)nnz, 0, end_bit,
                                                stream));
        void* temp = sort_scratch.take<unsigned char>(bytes);
        if ((st = sort_scratch.commit())) return st;
        OB_CUDA(cub::DeviceRadixSort::SortPairs(temp, bytes, keys, sorted, index, perm, (int)nnz, 0, end_bit, stream));
        dev_transpose_place_kernel<<<grid_of(nnz), kThreads, 0, stream>>>(nnz, sorted, perm, M.val, M.rows, col, val);
        OB_CHECK_LAUNCH("amg device build: transpose place");
    }
    if ((st = exclusive_scan(count, off, M.cols, stream))) return st;
    *out = DevCsr{M.cols, M.rows, nnz, off, col, val};
    return OB_OK;
}

// Levels of the hierarchy of the n x n operator (device CSR, float64) built on the device while
// a level has at least min_rows rows (and the host's stopping rules do not end it): aggregate()
// (strength, MIS-2 rounds, two hops of the label spread, aggregate sizes), damped_diagonal() (the
// power steps on the device, the growth summed on the host in row order), prolongator(),
// transpose() and galerkin(), each level's arithmetic as the host's.
int build_device_levels(const DevCsr& fine, uint32_t seed, int min_rows, DevBuild* B, cudaStream_t stream) {
    int st = OB_OK;
    DevCsr A = fine;
    const int* weights = nullptr;  // device, the current level's row weights (null: every row 1)
    std::vector<int> host_weights;
    while (true) {
        const int n = A.rows;
        if (n < min_rows || n <= kMaxCoarse || (int)B->levels.size() + 1 >= kMaxLevels) {
            // Below min_rows the host takes over (it stops at once where the rules end here).
            B->stopped = n <= kMaxCoarse || (int)B->levels.size() + 1 >= kMaxLevels;
            B->levels.push_back(DevLevel{A});
            break;
        }
        Scratch scratch(stream);
        double* l1 = scratch.take<double>(n);
        double* scaled = scratch.take<double>(n);
        uint32_t* priority = scratch.take<uint32_t>(n);
        int* state = scratch.take<int>(n);
        int* next = scratch.take<int>(n);
        int64_t* key = scratch.take<int64_t>(n);
        int* undecided = scratch.take<int>(1);
        int* flags = scratch.take<int>((size_t)n + 1);
        int* scan = scratch.take<int>((size_t)n + 1);
        int* label0 = scratch.take<int>(n);
        int* hop = scratch.take<int>(n);
        double* x = scratch.take<double>(n);
        double* y = scratch.take<double>(n);
        long long* count = scratch.take<long long>((size_t)n + 1);
        long long* raw = scratch.take<long long>((size_t)n + 1);
        if ((st = scratch.commit())) return st;
        int* label = nullptr;
        double* damped = nullptr;
        if ((st = keep_alloc(B, &label, n, stream)) || (st = keep_alloc(B, &damped, n, stream))) return st;
        const int grid = grid_of(n);
        dev_setup_kernel<<<grid, kThreads, 0, stream>>>(n, A.off, A.col, A.val, seed, l1, scaled, priority, state);
        OB_CHECK_LAUNCH("amg device build: setup");
        for (int round = 0; round < kMisRounds; ++round) {
            OB_CUDA(cudaMemsetAsync(undecided, 0, sizeof(int), stream));
            dev_mis_keys_kernel<<<grid, kThreads, 0, stream>>>(n, A.off, A.col, A.val, scaled, state, priority, key);
            OB_CHECK_LAUNCH("amg device build: MIS keys");
            dev_mis_decide_kernel<<<grid, kThreads, 0, stream>>>(n, A.off, A.col, A.val, scaled, state, priority, key,
                                                                  next, undecided);
            OB_CHECK_LAUNCH("amg device build: MIS decide");
            std::swap(state, next);
            const int left = read_one(undecided, stream, &st);
            if (st) return st;
            if (left == 0) break;
        }
        OB_CUDA(cudaMemsetAsync(flags + n, 0, sizeof(int), stream));
        dev_root_flags_kernel<<<grid, kThreads, 0, stream>>>(n, state, flags);
        OB_CHECK_LAUNCH("amg device build: root flags");
        if ((st = exclusive_scan(flags, scan, n, stream))) return st;
        const int n_aggregates = read_one(scan + n, stream, &st);
        if (st) return st;
        if (n_aggregates == 0 || n_aggregates >= kMinCoarsening * n) {
            B->stopped = true;
            B->levels.push_back(DevLevel{A});
            break;
        }
        dev_first_labels_kernel<<<grid, kThreads, 0, stream>>>(n, flags, scan, label0);
        dev_spread_kernel<<<grid, kThreads, 0, stream>>>(n, A.off, A.col, A.val, scaled, label0, hop);
        dev_spread_kernel<<<grid, kThreads, 0, stream>>>(n, A.off, A.col, A.val, scaled, hop, label);
        OB_CHECK_LAUNCH("amg device build: labels");
        int* sizes = nullptr;
        if ((st = keep_alloc(B, &sizes, n_aggregates, stream))) return st;
        OB_CUDA(cudaMemsetAsync(sizes, 0, sizeof(int) * n_aggregates, stream));
        dev_sizes_kernel<<<grid, kThreads, 0, stream>>>(n, label, weights, sizes);
        OB_CHECK_LAUNCH("amg device build: sizes");
        // omega from the power steps' growth, summed on the host in row order.
        dev_signs_kernel<<<grid, kThreads, 0, stream>>>(n, seed, x);
        for (int step = 0; step < kPowerSteps; ++step) {
            dev_power_kernel<<<grid, kThreads, 0, stream>>>(n, A.off, A.col, A.val, l1, x, y);
            std::swap(x, y);
        }
        OB_CHECK_LAUNCH("amg device build: power steps");
        std::vector<double> host_x(n);
        OB_CUDA(cudaMemcpyAsync(host_x.data(), x, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
        OB_CUDA(cudaStreamSynchronize(stream));
        double growth = 0.0;
        for (int i = 0; i < n; ++i) growth += host_x[i] * host_x[i];
        double rho = 1.0;
        if (growth > 0.0 && std::isfinite(growth)) rho = std::pow(std::sqrt(growth / (double)n), 1.0 / kPowerSteps);
        dev_damped_kernel<<<grid, kThreads, 0, stream>>>(n, l1, kJacobiFactor / rho, damped);
        OB_CHECK_LAUNCH("amg device build: damped diagonal");
        // P, R = P^T, then A P and R (A P).
        DevCsr P, R, AP, coarse;
        OB_CUDA(cudaMemsetAsync(count + n, 0, sizeof(long long), stream));
        dev_prolongator_kernel<false><<<grid, kThreads, 0, stream>>>(n, n_aggregates, A.off, A.col, A.val, label,
                                                                     weights, sizes, damped, count, nullptr, nullptr,
                                                                     nullptr);
        OB_CHECK_LAUNCH("amg device build: prolongator counts");
        st = assemble(n, n_aggregates, count,
                      [&](const long long* start, unsigned long long* keys, double* values) {
                          dev_prolongator_kernel<true><<<grid, kThreads, 0, stream>>>(
                              n, n_aggregates, A.off, A.col, A.val, label, weights, sizes, damped, nullptr, start, keys,
                              values);
                      },
                      B, &P, stream);
        if (st || (st = transpose_device(P, B, &R, stream))) return st;
        // galerkin(): the key budget of each product (every contribution counted) against the
        // fallback's cap.
        const long long budget = kTripletFactor * (A.nnz + n);
        const bool capped = (long long)n * n_aggregates > kDenseOutputCap;
        Scratch sums(stream);
        long long* total = sums.take<long long>(1);
        size_t reduce_bytes = 0;
        OB_CUDA(cub::DeviceReduce::Sum(nullptr, reduce_bytes, raw, total, n, stream));
        void* reduce_temp = sums.take<unsigned char>(reduce_bytes);
        if ((st = sums.commit())) return st;
        OB_CUDA(cudaMemsetAsync(count + n, 0, sizeof(long long), stream));
        dev_product_kernel<false><<<grid, kThreads, 0, stream>>>(n, n_aggregates, A.off, A.col, A.val, P.off, P.col,
                                                                 P.val, count, raw, nullptr, nullptr, nullptr);
        OB_CHECK_LAUNCH("amg device build: A P counts");
        OB_CUDA(cub::DeviceReduce::Sum(reduce_temp, reduce_bytes, raw, total, n, stream));
        const long long ap_contributions = read_one(total, stream, &st);
        if (st) return st;
        if (ap_contributions > budget && capped) {
            B->stopped = true;
            B->levels.push_back(DevLevel{A});
            break;
        }
        st = assemble(n, n_aggregates, count,
                      [&](const long long* start, unsigned long long* keys, double* values) {
                          dev_product_kernel<true><<<grid, kThreads, 0, stream>>>(
                              n, n_aggregates, A.off, A.col, A.val, P.off, P.col, P.val, nullptr, nullptr, start, keys,
                              values);
                      },
                      B, &AP, stream);
        if (st) return st;
        const int nc = n_aggregates;
        Scratch rap(stream);
        long long* ccount = rap.take<long long>((size_t)nc + 1);
        long long* craw = rap.take<long long>((size_t)nc + 1);
        size_t cbytes = 0;
        OB_CUDA(cub::DeviceReduce::Sum(nullptr, cbytes, craw, total, nc, stream));
        void* ctemp = rap.take<unsigned char>(cbytes);
        if ((st = rap.commit())) return st;
        OB_CUDA(cudaMemsetAsync(ccount + nc, 0, sizeof(long long), stream));
        dev_product_kernel<false><<<grid_of(nc), kThreads, 0, stream>>>(nc, nc, R.off, R.col, R.val, AP.off, AP.col,
                                                                        AP.val, ccount, craw, nullptr, nullptr, nullptr);
        OB_CHECK_LAUNCH("amg device build: R A P counts");
        OB_CUDA(cub::DeviceReduce::Sum(ctemp, cbytes, craw, total, nc, stream));
        const long long rap_contributions = read_one(total, stream, &st);
        if (st) return st;
        if (rap_contributions > budget && capped) {
            B->stopped = true;
            B->levels.push_back(DevLevel{A});
            break;
        }
        st = assemble(nc, nc, ccount,
                      [&](const long long* start, unsigned long long* keys, double* values) {
                          dev_product_kernel<true><<<grid_of(nc), kThreads, 0, stream>>>(
                              nc, nc, R.off, R.col, R.val, AP.off, AP.col, AP.val, nullptr, nullptr, start, keys,
                              values);
                      },
                      B, &coarse, stream);
        if (st) return st;
        B->levels.push_back(DevLevel{A, P, R, damped});
        weights = sizes;
        host_weights.assign(nc, 0);
        OB_CUDA(cudaMemcpyAsync(host_weights.data(), sizes, sizeof(int) * nc, cudaMemcpyDeviceToHost, stream));
        OB_CUDA(cudaStreamSynchronize(stream));
        A = coarse;
    }
    B->weights = std::move(host_weights);
    return OB_OK;
}

void release_build(DevBuild* B) {
    for (void* p : B->owned) cudaFree(p);
    B->owned.clear();
}

__global__ void dev_narrow_kernel(long long n, const double* __restrict__ in, float* __restrict__ out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}

__global__ void dev_jacobi_kernel(int n, const int* __restrict__ off, const int* __restrict__ col,
                                  const double* __restrict__ val, float* __restrict__ jacobi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 0.0;
    for (int k = off[i]; k < off[i + 1]; ++k)
        if (col[k] == i) d += val[k];
    jacobi[i] = (float)inverse_or_one(d);
}

HCsr download(const DevCsr& M, cudaStream_t stream, int* status) {
    HCsr H;
    H.rows = M.rows;
    H.cols = M.cols;
    H.off.resize((size_t)M.rows + 1);
    H.col.resize((size_t)M.nnz);
    H.val.resize((size_t)M.nnz);
    cudaError_t e = cudaMemcpyAsync(H.off.data(), M.off, sizeof(int) * H.off.size(), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && M.nnz)
        e = cudaMemcpyAsync(H.col.data(), M.col, sizeof(int) * (size_t)M.nnz, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && M.nnz)
        e = cudaMemcpyAsync(H.val.data(), M.val, sizeof(double) * (size_t)M.nnz, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) *status = cuda_status(e, "amg device build: download");
    return H;
}

// ---------------------------------------------------------------------------------------------
// Device
// ---------------------------------------------------------------------------------------------

struct DeviceLevel {
    int n = 0;
    long long nnz = 0;
    int* off = nullptr;
    int* col = nullptr;
    float* val = nullptr;
    float* damped = nullptr;
    int n_coarse = 0;
    long long pnnz = 0, rnnz = 0;  // stored entries of the prolongation and the restriction
    int *poff = nullptr, *pcol = nullptr, *roff = nullptr, *rcol = nullptr;
    float *pval = nullptr, *rval = nullptr;
};

struct ColumnState {
    double rho, alpha, beta, rr, bnorm2, res2, scale;
    int active, inner_done, outer_done, status, iters;
};

struct LoopState {
    int iter, max_inner, any_active, pad;
    double inner_tol2;
};

struct Work {
    int kp = 0, G = 0;
    std::vector<float*> b, x, y, r;  // per level (level 0 has no b and x: its input and output are res and z)
    float *d = nullptr, *res = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
    double *b64 = nullptr, *x64 = nullptr, *r64 = nullptr;
    double* partials = nullptr;  // [blocks][kp]
    unsigned int* counters = nullptr;
    ColumnState* cols = nullptr;
    ColumnState* host_cols = nullptr;
    LoopState* loop = nullptr;
    int blocks = 0;
    cudaGraphExec_t inner = nullptr;
    cudaGraph_t inner_graph = nullptr;
    cudaGraphExec_t round = nullptr;
    cudaGraph_t round_graph = nullptr;
    int inner_launches = 0, round_launches = 0;
    std::vector<void*> allocations;
};

struct Amg {
    int n = 0;
    long long nnz = 0;
    const int* off64 = nullptr;
    const int* col64 = nullptr;
    const double* val64 = nullptr;
    std::vector<DeviceLevel> levels;
    int coarse_rows = 0, n_active = 0;
    float* inverse = nullptr;
    int* slots = nullptr;  // coarsest row -> active slot or -1
    float* jacobi = nullptr;
    bool usable = false;
    std::vector<void*> allocations;
    std::vector<std::unique_ptr<Work>> work;
    cudaStream_t capture = nullptr;
    std::mutex lock;
};

template <typename T>
int upload(Amg* M, const std::vector<T>& host, T** out, cudaStream_t stream) {
    *out = nullptr;
    if (host.empty()) return OB_OK;
    void* p = nullptr;
    (void)stream;
    OB_CUDA(cudaMalloc(&p, sizeof(T) * host.size()));
    M->allocations.push_back(p);
    OB_CUDA(cudaMemcpy(p, host.data(), sizeof(T) * host.size(), cudaMemcpyHostToDevice));
    *out = static_cast<T*>(p);
    return OB_OK;
}

std::vector<float> narrow(const std::vector<double>& v) {
    std::vector<float> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = (float)v[i];
    return out;
}

void release_work(Work* W) {
    if (W->inner) cudaGraphExecDestroy(W->inner);
    if (W->inner_graph) cudaGraphDestroy(W->inner_graph);
    if (W->round) cudaGraphExecDestroy(W->round);
    if (W->round_graph) cudaGraphDestroy(W->round_graph);
    if (W->host_cols) cudaFreeHost(W->host_cols);
    for (void* p : W->allocations) cudaFree(p);
    W->allocations.clear();
}

void release(Amg* M) {
    for (auto& W : M->work) release_work(W.get());
    M->work.clear();
    for (void* p : M->allocations) cudaFree(p);
    M->allocations.clear();
    if (M->capture) cudaStreamDestroy(M->capture);
}

// ---- kernels ----------------------------------------------------------------------------------

__device__ __forceinline__ float4 f4(float v) { return make_float4(v, v, v, v); }
__device__ __forceinline__ void fma4(float a, const float4& v, float4& acc) {
    acc.x = fmaf(a, v.x, acc.x);
    acc.y = fmaf(a, v.y, acc.y);
    acc.z = fmaf(a, v.z, acc.z);
    acc.w = fmaf(a, v.w, acc.w);
}

// Row `row` of M x over a row group: lane reads columns [4 lane, 4 lane + 4).
__device__ __forceinline__ float4 row_product(const int* __restrict__ off, const int* __restrict__ col,
                                              const float* __restrict__ val,
                                              const float4* __restrict__ x, int G, int row,
                                              int lane) {
    float4 acc = f4(0.0f);
    const int end = off[row + 1];
    int e = off[row];
    for (; e + 1 < end; e += 2) {
        const int j0 = col[e], j1 = col[e + 1];
        const float a0 = val[e], a1 = val[e + 1];
        const float4 v0 = x[(size_t)j0 * G + lane];
        const float4 v1 = x[(size_t)j1 * G + lane];
        fma4(a0, v0, acc);
        fma4(a1, v1, acc);
    }
    if (e < end) fma4(val[e], x[(size_t)col[e] * G + lane], acc);
    return acc;
}

// Per-thread column partial sums (4 columns a lane) -> block partials[block][kp] (fixed tree).
__device__ __forceinline__ void store_column_partials(double4 mine, int G, double* partials,
                                                      double* smem) {
    // smem: [groups][kp] doubles; groups = blockDim / G.
    const int lane = threadIdx.x % G, group = threadIdx.x / G, kp = 4 * G;
    const int groups = blockDim.x / G;
    double* slot = smem + (size_t)group * kp + 4 * lane;
    slot[0] = mine.x;
    slot[1] = mine.y;
    slot[2] = mine.z;
    slot[3] = mine.w;
    __syncthreads();
    for (int c = threadIdx.x; c < kp; c += blockDim.x) {
        double s = 0.0;
        for (int g = 0; g < groups; ++g) s += smem[(size_t)g * kp + c];
        partials[(size_t)blockIdx.x * kp + c] = s;
    }
    // Every writer publishes its partials before the block takes its last-block ticket.
    __threadfence();
}

// Last block: sums partials[blocks][kp] per column in block order into smem[kp].
__device__ __forceinline__ void fold_columns(const double* partials, int blocks, int kp, double* smem) {
    const int subsets = blockDim.x / kp;  // kp divides blockDim (both powers of two, kp <= 128)
    const int c = threadIdx.x % kp, s = threadIdx.x / kp;
    double sum = 0.0;
    for (int b = s; b < blocks; b += subsets) sum += partials[(size_t)b * kp + c];
    __syncthreads();
    smem[threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.x < kp) {
        double total = 0.0;
        for (int t = 0; t < subsets; ++t) total += smem[t * kp + threadIdx.x];
        smem[blockDim.x + threadIdx.x] = total;
    }
    __syncthreads();
}

// x = d .* b (the first sweep from zero, or the Jacobi preconditioner); with `cols`, also the
// column dots b.x folded into cols[c].rho (top level: r.z) with beta.
template <bool kDot>
__global__ void __launch_bounds__(kThreads) scale_kernel(int n, int G, const float* __restrict__ d,
                                                         const float4* __restrict__ b, float4* __restrict__ x,
                                                         double* partials, unsigned int* counter,
                                                         ColumnState* cols) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x % G, groups = blockDim.x / G;
    double4 mine = make_double4(0, 0, 0, 0);
    for (int row = blockIdx.x * groups + threadIdx.x / G; row < n; row += gridDim.x * groups) {
        const float s = d[row];
        const float4 v = b[(size_t)row * G + lane];
        const float4 o = make_float4(s * v.x, s * v.y, s * v.z, s * v.w);
        x[(size_t)row * G + lane] = o;
        if (kDot) {
            mine.x += (double)v.x * o.x;
            mine.y += (double)v.y * o.y;
            mine.z += (double)v.z * o.z;
            mine.w += (double)v.w * o.w;
        }
    }
    if (!kDot) return;
    store_column_partials(mine, G, partials, smem);
    __shared__ int last;
    if (!last_block_arrived(counter, &last)) return;
    const int kp = 4 * G;
    fold_columns(partials, gridDim.x, kp, smem);
    if (threadIdx.x < kp) {
        ColumnState& C = cols[threadIdx.x];
        const double rho = smem[blockDim.x + threadIdx.x];
        if (C.active) {
            C.beta = (C.rho != 0.0) ? rho / C.rho : 0.0;
            C.rho = rho;
        } else {
            C.beta = 0.0;
        }
    }
}

// One damped-Jacobi sweep x_out = x_in + d .* (b - A x_in); kDot adds the top level's r.z fold.
template <bool kDot>
__global__ void __launch_bounds__(kThreads) sweep_kernel(int n, int G, const int* __restrict__ off,
                                                         const int* __restrict__ col,
                                                         const float* __restrict__ val,
                                                         const float* __restrict__ d,
                                                         const float4* __restrict__ b,
                                                         const float4* __restrict__ x_in,
                                                         float4* __restrict__ x_out, double* partials,
                                                         unsigned int* counter, ColumnState* cols) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x % G, groups = blockDim.x / G;
    double4 mine = make_double4(0, 0, 0, 0);
    for (int row = blockIdx.x * groups + threadIdx.x / G; row < n; row += gridDim.x * groups) {
        const float4 ax = row_product(off, col, val, x_in, G, row, lane);
        const float4 bv = b[(size_t)row * G + lane];
        const float4 xv = x_in[(size_t)row * G + lane];
        const float s = d[row];
        float4 o;
        o.x = fmaf(s, bv.x - ax.x, xv.x);
        o.y = fmaf(s, bv.y - ax.y, xv.y);
        o.z = fmaf(s, bv.z - ax.z, xv.z);
        o.w = fmaf(s, bv.w - ax.w, xv.w);
        x_out[(size_t)row * G + lane] = o;
        if (kDot) {
            mine.x += (double)bv.x * o.x;
            mine.y += (double)bv.y * o.y;
            mine.z += (double)bv.z * o.z;
            mine.w += (double)bv.w * o.w;
        }
    }
    if (!kDot) return;
    store_column_partials(mine, G, partials, smem);
    __shared__ int last;
    if (!last_block_arrived(counter, &last)) return;
    const int kp = 4 * G;
    fold_columns(partials, gridDim.x, kp, smem);
    if (threadIdx.x < kp) {
        ColumnState& C = cols[threadIdx.x];
        const double rho = smem[blockDim.x + threadIdx.x];
        if (C.active) {
            C.beta = (C.rho != 0.0) ? rho / C.rho : 0.0;
            C.rho = rho;
        } else {
            C.beta = 0.0;
        }
    }
}

// The column dots b.x folded into rho and beta (the top level's r.z after a coarse solve).
__global__ void __launch_bounds__(kThreads) column_dot_kernel(int n, int G, const float4* __restrict__ b,
                                                              const float4* __restrict__ x, double* partials,
                                                              unsigned int* counter, ColumnState* cols) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x % G, groups = blockDim.x / G;
    double4 mine = make_double4(0, 0, 0, 0);
    for (int row = blockIdx.x * groups + threadIdx.x / G; row < n; row += gridDim.x * groups) {
        const float4 v = b[(size_t)row * G + lane], o = x[(size_t)row * G + lane];
        mine.x += (double)v.x * o.x;
        mine.y += (double)v.y * o.y;
        mine.z += (double)v.z * o.z;
        mine.w += (double)v.w * o.w;
    }
    store_column_partials(mine, G, partials, smem);
    __shared__ int last;
    if (!last_block_arrived(counter, &last)) return;
    const int kp = 4 * G;
    fold_columns(partials, gridDim.x, kp, smem);
    if (threadIdx.x < kp) {
        ColumnState& C = cols[threadIdx.x];
        const double rho = smem[blockDim.x + threadIdx.x];
        if (C.active) {
            C.beta = (C.rho != 0.0) ? rho / C.rho : 0.0;
            C.rho = rho;
        } else {
            C.beta = 0.0;
        }
    }
}

// r = b - A x.
__global__ void __launch_bounds__(kThreads) residual_kernel(int n, int G, const int* __restrict__ off,
                                                            const int* __restrict__ col,
                                                            const float* __restrict__ val,
                                                            const float4* __restrict__ b,
                                                            const float4* __restrict__ x,
                                                            float4* __restrict__ r) {
    const int lane = threadIdx.x % G, groups = blockDim.x / G;
    for (int row = blockIdx.x * groups + threadIdx.x / G; row < n; row += gridDim.x * groups) {
        const float4 ax = row_product(off, col, val, x, G, row, lane);
        const float4 bv = b[(size_t)row * G + lane];
        r[(size_t)row * G + lane] = make_float4(bv.x - ax.x, bv.y - ax.y, bv.z - ax.z, bv.w - ax.w);
    }
}

// y = M x (kAccumulate: y += M x), M rectangular (restriction or prolongation).
template <bool kAccumulate>
__global__ void __launch_bounds__(kThreads) spmm_kernel(int rows, int G, const int* __restrict__ off,
                                                        const int* __restrict__ col,
                                                        const float* __restrict__ val,
                                                        const float4* __restrict__ x,
                                                        float4* __restrict__ y) {
    const int lane = threadIdx.x % G, groups = blockDim.x / G;
    for (int row = blockIdx.x * groups + threadIdx.x / G; row < rows; row += gridDim.x * groups) {
        float4 v = row_product(off, col, val, x, G, row, lane);
        if (kAccumulate) {
            const float4 o = y[(size_t)row * G + lane];
            v.x += o.x;
            v.y += o.y;
            v.z += o.z;
            v.w += o.w;
        }
        y[(size_t)row * G + lane] = v;
    }
}

// Coarsest level: x = S^+ b over the active rows (inactive rows solve to zero). One block a row.
__global__ void __launch_bounds__(kThreads) coarse_kernel(int rows, int G, int m, const float* __restrict__ inverse,
                                                          const int* __restrict__ slots,
                                                          const int* __restrict__ active,
                                                          const float4* __restrict__ b,
                                                          float4* __restrict__ x) {
    extern __shared__ double smem[];
    const int row = blockIdx.x;
    const int lane = threadIdx.x % G, part = threadIdx.x / G, parts = blockDim.x / G;
    const int slot = slots[row];
    float4 acc = f4(0.0f);
    if (slot >= 0)
        for (int t = part; t < m; t += parts) fma4(inverse[(size_t)slot * m + t], b[(size_t)active[t] * G + lane], acc);
    float* fs = reinterpret_cast<float*>(smem);
    reinterpret_cast<float4*>(fs)[threadIdx.x] = acc;
    __syncthreads();
    if (part == 0) {
        float4 total = f4(0.0f);
        for (int p = 0; p < parts; ++p) {
            const float4 v = reinterpret_cast<float4*>(fs)[p * G + lane];
            total.x += v.x;
            total.y += v.y;
            total.z += v.z;
            total.w += v.w;
        }
        x[(size_t)row * G + lane] = total;
    }
}

// q = A z + beta q, p = z + beta p (the CG direction update folded into the product), and the
// column dots p.q folded into alpha = rho / p.q by the last block.
__global__ void __launch_bounds__(kThreads) direction_kernel(int n, int G, const int* __restrict__ off,
                                                             const int* __restrict__ col,
                                                             const float* __restrict__ val,
                                                             const float4* __restrict__ z,
                                                             float4* __restrict__ p, float4* __restrict__ q,
                                                             double* partials, unsigned int* counter,
                                                             ColumnState* cols) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x % G, groups = blockDim.x / G;
    const float4 beta = make_float4((float)cols[4 * lane].beta, (float)cols[4 * lane + 1].beta,
                                    (float)cols[4 * lane + 2].beta, (float)cols[4 * lane + 3].beta);
    double4 mine = make_double4(0, 0, 0, 0);
    for (int row = blockIdx.x * groups + threadIdx.x / G; row < n; row += gridDim.x * groups) {
        const float4 az = row_product(off, col, val, z, G, row, lane);
        const size_t at = (size_t)row * G + lane;
        const float4 zv = z[at], pv = p[at], qv = q[at];
        float4 pn, qn;
        pn.x = fmaf(beta.x, pv.x, zv.x);
        pn.y = fmaf(beta.y, pv.y, zv.y);
        pn.z = fmaf(beta.z, pv.z, zv.z);
        pn.w = fmaf(beta.w, pv.w, zv.w);
        qn.x = fmaf(beta.x, qv.x, az.x);
        qn.y = fmaf(beta.y, qv.y, az.y);
        qn.z = fmaf(beta.z, qv.z, az.z);
        qn.w = fmaf(beta.w, qv.w, az.w);
        p[at] = pn;
        q[at] = qn;
        mine.x += (double)pn.x * qn.x;
        mine.y += (double)pn.y * qn.y;
        mine.z += (double)pn.z * qn.z;
        mine.w += (double)pn.w * qn.w;
    }
    store_column_partials(mine, G, partials, smem);
    __shared__ int last;
    if (!last_block_arrived(counter, &last)) return;
    const int kp = 4 * G;
    fold_columns(partials, gridDim.x, kp, smem);
    if (threadIdx.x < kp) {
        ColumnState& C = cols[threadIdx.x];
        const double pq = smem[blockDim.x + threadIdx.x];
        C.alpha = 0.0;
        if (C.active) {
            if (pq > 0.0 && std::isfinite(pq) && std::isfinite(C.rho)) {
                C.alpha = C.rho / pq;
            } else {
                // A direction of no curvature: the column has converged as far as it can.
                C.active = 0;
                if (!std::isfinite(pq) || !std::isfinite(C.rho)) C.status = OB_STATUS_NONFINITE;
            }
        }
    }
}

// d += alpha p, r -= alpha q; the column dots r.r decide which columns stay active.
__global__ void __launch_bounds__(kThreads) update_kernel(int n, int G, const float4* __restrict__ p,
                                                          const float4* __restrict__ q,
                                                          float4* __restrict__ d, float4* __restrict__ r,
                                                          double* partials, unsigned int* counter,
                                                          ColumnState* cols, LoopState* loop) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x % G, groups = blockDim.x / G;
    const float4 alpha = make_float4((float)cols[4 * lane].alpha, (float)cols[4 * lane + 1].alpha,
                                     (float)cols[4 * lane + 2].alpha, (float)cols[4 * lane + 3].alpha);
    double4 mine = make_double4(0, 0, 0, 0);
    for (int row = blockIdx.x * groups + threadIdx.x / G; row < n; row += gridDim.x * groups) {
        const size_t at = (size_t)row * G + lane;
        const float4 pv = p[at], qv = q[at];
        float4 dv = d[at], rv = r[at];
        dv.x = fmaf(alpha.x, pv.x, dv.x);
        dv.y = fmaf(alpha.y, pv.y, dv.y);
        dv.z = fmaf(alpha.z, pv.z, dv.z);
        dv.w = fmaf(alpha.w, pv.w, dv.w);
        rv.x = fmaf(-alpha.x, qv.x, rv.x);
        rv.y = fmaf(-alpha.y, qv.y, rv.y);
        rv.z = fmaf(-alpha.z, qv.z, rv.z);
        rv.w = fmaf(-alpha.w, qv.w, rv.w);
        d[at] = dv;
        r[at] = rv;
        mine.x += (double)rv.x * rv.x;
        mine.y += (double)rv.y * rv.y;
        mine.z += (double)rv.z * rv.z;
        mine.w += (double)rv.w * rv.w;
    }
    store_column_partials(mine, G, partials, smem);
    __shared__ int last;
    if (!last_block_arrived(counter, &last)) return;
    const int kp = 4 * G;
    fold_columns(partials, gridDim.x, kp, smem);
    if (threadIdx.x < kp) {
        ColumnState& C = cols[threadIdx.x];
        const double rr = smem[blockDim.x + threadIdx.x];
        if (C.active) {
            C.rr = rr;
            C.iters += 1;
            if (!std::isfinite(rr)) {
                C.active = 0;
                C.status = OB_STATUS_NONFINITE;
            } else if (rr <= loop->inner_tol2) {
                C.active = 0;
            }
        }
    }
}

// Ends a loop body: counts the iteration and continues while a column is active.
__global__ void decide_kernel(ColumnState* cols, int kp, LoopState* loop,
                              cudaGraphConditionalHandle handle) {
    int any = 0;
    for (int c = threadIdx.x; c < kp; c += blockDim.x) any |= cols[c].active;
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        loop->iter += 1;
        loop->any_active = any;
        const bool go = any && loop->iter < loop->max_inner;
        cudaGraphSetConditional(handle, go ? 1u : 0u);
    }
}

// ---- float64 refinement kernels ----------------------------------------------------------------

// The caller's [n][ld] float64 rows (k live columns) -> [n][kp] float64 (pad columns zero).
__global__ void gather_columns_kernel(int n, int k, int kp, const double* __restrict__ in, long long ld,
                                      double* __restrict__ out) {
    const long long total = (long long)n * kp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(t / kp), c = (int)(t % kp);
        out[t] = c < k ? in[(size_t)row * ld + c] : 0.0;
    }
}

__global__ void scatter_columns_kernel(int n, int k, int kp, const double* __restrict__ in,
                                       double* __restrict__ out, long long ld) {
    const long long total = (long long)n * k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(t / k), c = (int)(t % k);
        out[(size_t)row * ld + c] = in[(size_t)row * kp + c];
    }
}

// Column norms |b|^2 into cols[c].bnorm2 and the column states reset for a solve.
__global__ void __launch_bounds__(kThreads) start_kernel(int n, int G, int k, const double* __restrict__ b,
                                                         double* partials, unsigned int* counter,
                                                         ColumnState* cols) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x % G, groups = blockDim.x / G;
    double4 mine = make_double4(0, 0, 0, 0);
    for (int row = blockIdx.x * groups + threadIdx.x / G; row < n; row += gridDim.x * groups) {
        const double* v = b + (size_t)row * 4 * G + 4 * lane;
        mine.x += v[0] * v[0];
        mine.y += v[1] * v[1];
        mine.z += v[2] * v[2];
        mine.w += v[3] * v[3];
    }
    store_column_partials(mine, G, partials, smem);
    __shared__ int last;
    if (!last_block_arrived(counter, &last)) return;
    const int kp = 4 * G;
    fold_columns(partials, gridDim.x, kp, smem);
    if (threadIdx.x < kp) {
        ColumnState C = {};
        C.bnorm2 = smem[blockDim.x + threadIdx.x];
        C.outer_done = threadIdx.x >= k;
        C.status = OB_STATUS_CAPPED;
        cols[threadIdx.x] = C;
    }
}

// r = b - A x in float64 (the caller's values), its column norms, the outer convergence test,
// and r scaled by 1/|r| into float32 for the inner solve (d, p, q cleared for it).
__global__ void __launch_bounds__(kThreads) refine_residual_kernel(
    int n, int G, const int* __restrict__ off, const int* __restrict__ col, const double* __restrict__ val,
    const double* __restrict__ b, const double* __restrict__ x, double* __restrict__ r64,
    double* partials, unsigned int* counter, ColumnState* cols, double tol2) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x % G, groups = blockDim.x / G, kp = 4 * G;
    double4 mine = make_double4(0, 0, 0, 0);
    for (int row = blockIdx.x * groups + threadIdx.x / G; row < n; row += gridDim.x * groups) {
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        for (int e = off[row]; e < off[row + 1]; ++e) {
            const double a = val[e];
            const double* xv = x + (size_t)col[e] * kp + 4 * lane;
            const double2 u = *reinterpret_cast<const double2*>(xv);
            const double2 w = *reinterpret_cast<const double2*>(xv + 2);
            a0 = fma(a, u.x, a0);
            a1 = fma(a, u.y, a1);
            a2 = fma(a, w.x, a2);
            a3 = fma(a, w.y, a3);
        }
        const double* bv = b + (size_t)row * kp + 4 * lane;
        double* rv = r64 + (size_t)row * kp + 4 * lane;
        rv[0] = bv[0] - a0;
        rv[1] = bv[1] - a1;
        rv[2] = bv[2] - a2;
        rv[3] = bv[3] - a3;
        mine.x += rv[0] * rv[0];
        mine.y += rv[1] * rv[1];
        mine.z += rv[2] * rv[2];
        mine.w += rv[3] * rv[3];
    }
    store_column_partials(mine, G, partials, smem);
    __shared__ int last;
    if (!last_block_arrived(counter, &last)) return;
    fold_columns(partials, gridDim.x, kp, smem);
    if (threadIdx.x < kp) {
        ColumnState& C = cols[threadIdx.x];
        const double res2 = smem[blockDim.x + threadIdx.x];
        C.res2 = res2;
        if (!C.outer_done) {
            if (!std::isfinite(res2)) {
                C.outer_done = 1;
                C.status = OB_STATUS_NONFINITE;
            } else if (res2 <= tol2 * C.bnorm2 || res2 == 0.0) {
                C.outer_done = 1;
                C.status = OB_STATUS_CONVERGED;
            }
        }
        C.active = !C.outer_done;
        C.scale = (C.active && res2 > 0.0) ? sqrt(res2) : 0.0;
        C.rho = 0.0;
        C.alpha = C.beta = 0.0;
        C.rr = 1.0;
    }
}

// r32 = r64 / scale (0 for inactive columns), d = p = q = 0.
__global__ void narrow_kernel(int n, int kp, const double* __restrict__ r64, const ColumnState* cols,
                              float* __restrict__ r, float* __restrict__ d, float* __restrict__ p,
                              float* __restrict__ q) {
    const long long total = (long long)n * kp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t % kp);
        const double s = cols[c].scale;
        r[t] = s > 0.0 ? (float)(r64[t] / s) : 0.0f;
        d[t] = 0.0f;
        p[t] = 0.0f;
        q[t] = 0.0f;
    }
}

// x += scale * d (float64 accumulation of the correction).
__global__ void correct_kernel(int n, int kp, const float* __restrict__ d, const ColumnState* cols,
                               double* __restrict__ x) {
    const long long total = (long long)n * kp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const double s = cols[(int)(t % kp)].scale;
        if (s > 0.0) x[t] += s * (double)d[t];
    }
}

// The caller's float64 [n][ld] rows <-> float32 [n][kp], for ob_amg_apply.
__global__ void to_f32_kernel(int n, int k, int kp, const double* __restrict__ in, long long ld,
                              float* __restrict__ out) {
    const long long total = (long long)n * kp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(t / kp), c = (int)(t % kp);
        out[t] = c < k ? (float)in[(size_t)row * ld + c] : 0.0f;
    }
}

__global__ void from_f32_kernel(int n, int k, int kp, const float* __restrict__ in, double* __restrict__ out,
                                long long ld) {
    const long long total = (long long)n * k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(t / k), c = (int)(t % k);
        out[(size_t)row * ld + c] = (double)in[(size_t)row * kp + c];
    }
}

// ---- host orchestration -----------------------------------------------------------------------

int grid_for(long long threads) {
    const long long cap = 8LL * sm_count();
    return (int)std::max(1LL, std::min(cap, (threads + kThreads - 1) / kThreads));
}

size_t partial_smem(int G) { return sizeof(double) * std::max(2 * kThreads, (kThreads / G) * 4 * G); }

int padded_columns(int k) {
    int kp = 4;
    while (kp < k) kp *= 2;
    return kp;
}

int ensure_work(Amg* M, int kp, Work** out, cudaStream_t stream) {
    for (auto& W : M->work)
        if (W->kp == kp) {
            *out = W.get();
            return OB_OK;
        }
    auto W = std::make_unique<Work>();
    W->kp = kp;
    W->G = kp / 4;
    auto alloc = [&](size_t bytes, void** p) -> int {
        OB_CUDA(cudaMalloc(p, std::max<size_t>(bytes, 16)));
        W->allocations.push_back(*p);
        return OB_OK;
    };
    int st;
    const size_t L = M->levels.size();
    W->b.assign(L, nullptr);
    W->x.assign(L, nullptr);
    W->y.assign(L, nullptr);
    W->r.assign(L, nullptr);
    for (size_t l = 0; l < L; ++l) {
        const size_t bytes = sizeof(float) * (size_t)M->levels[l].n * kp;
        if (l > 0 && ((st = alloc(bytes, (void**)&W->b[l])) || (st = alloc(bytes, (void**)&W->x[l]))))
            return st;
        if ((st = alloc(bytes, (void**)&W->y[l])) || (st = alloc(bytes, (void**)&W->r[l]))) return st;
    }
    const size_t f = sizeof(float) * (size_t)M->n * kp, dd = sizeof(double) * (size_t)M->n * kp;
    if ((st = alloc(f, (void**)&W->d)) || (st = alloc(f, (void**)&W->res)) || (st = alloc(f, (void**)&W->z)) ||
        (st = alloc(f, (void**)&W->p)) || (st = alloc(f, (void**)&W->q)) || (st = alloc(dd, (void**)&W->b64)) ||
        (st = alloc(dd, (void**)&W->x64)) || (st = alloc(dd, (void**)&W->r64)))
        return st;
    W->blocks = 2 * sm_count();
    if ((st = alloc(sizeof(double) * (size_t)W->blocks * kp, (void**)&W->partials)) ||
        (st = alloc(sizeof(unsigned int) * 8, (void**)&W->counters)) ||
        (st = alloc(sizeof(ColumnState) * kp, (void**)&W->cols)) ||
        (st = alloc(sizeof(LoopState), (void**)&W->loop)))
        return st;
    OB_CUDA(cudaMemsetAsync(W->counters, 0, sizeof(unsigned int) * 8, stream));
    OB_CUDA(cudaMallocHost((void**)&W->host_cols, sizeof(ColumnState) * kp));
    *out = W.get();
    M->work.push_back(std::move(W));
    return OB_OK;
}

// Enqueues the V-cycle below level l: out = M_l b. At the top (l == 0, top_dot) the last
// post-sweep also folds r.z (= b.out) into the column states. Returns the launches enqueued.
int enqueue_cycle(Amg* M, Work* W, size_t l, const float* b, float* out, bool top_dot,
                  cudaStream_t stream, int* launches) {
    const int G = W->G;
    const size_t smem = partial_smem(G);
    const DeviceLevel& L = M->levels[l];
    auto f4p = [](const float* p) { return reinterpret_cast<const float4*>(p); };
    auto f4m = [](float* p) { return reinterpret_cast<float4*>(p); };
    if (!M->usable) {
        // No usable hierarchy: the Jacobi preconditioner (ordito/linalg.py:5118-5119).
        if (top_dot)
            scale_kernel<true><<<W->blocks, kThreads, smem, stream>>>(L.n, G, M->jacobi, f4p(b), f4m(out),
                                                                      W->partials, W->counters + 0, W->cols);
        else
            scale_kernel<false><<<grid_for((long long)L.n * G), kThreads, smem, stream>>>(
                L.n, G, M->jacobi, f4p(b), f4m(out), nullptr, nullptr, nullptr);
        OB_CHECK_LAUNCH("amg jacobi");
        ++*launches;
        return OB_OK;
    }
    if (l + 1 == M->levels.size()) {
        coarse_kernel<<<L.n, kThreads, sizeof(float4) * kThreads, stream>>>(
            L.n, G, M->n_active, M->inverse, M->slots, M->slots + L.n, f4p(b), f4m(out));
        OB_CHECK_LAUNCH("amg coarse");
        ++*launches;
        if (top_dot) {
            column_dot_kernel<<<W->blocks, kThreads, smem, stream>>>(L.n, G, f4p(b), f4p(out), W->partials,
                                                                      W->counters + 0, W->cols);
            OB_CHECK_LAUNCH("amg coarse dot");
            ++*launches;
        }
        return OB_OK;
    }
    const int grid = grid_for((long long)L.n * G);
    float* other = W->y[l];
    // Pre-smoothing: the first sweep from zero is a write; the second lands in `out`.
    scale_kernel<false><<<grid, kThreads, 0, stream>>>(L.n, G, L.damped, f4p(b), f4m(other), nullptr,
                                                         nullptr, nullptr);
    OB_CHECK_LAUNCH("amg first sweep");
    sweep_kernel<false><<<grid, kThreads, 0, stream>>>(L.n, G, L.off, L.col, L.val, L.damped, f4p(b),
                                                        f4p(other), f4m(out), nullptr, nullptr, nullptr);
    OB_CHECK_LAUNCH("amg sweep");
    residual_kernel<<<grid, kThreads, 0, stream>>>(L.n, G, L.off, L.col, L.val, f4p(b), f4p(out), f4m(W->r[l]));
    OB_CHECK_LAUNCH("amg residual");
    const DeviceLevel& C = M->levels[l + 1];
    spmm_kernel<false><<<grid_for((long long)C.n * G), kThreads, 0, stream>>>(
        C.n, G, L.roff, L.rcol, L.rval, f4p(W->r[l]), f4m(W->b[l + 1]));
    OB_CHECK_LAUNCH("amg restrict");
    *launches += 4;
    int st = enqueue_cycle(M, W, l + 1, W->b[l + 1], W->x[l + 1], false, stream, launches);
    if (st) return st;
    spmm_kernel<true><<<grid, kThreads, 0, stream>>>(L.n, G, L.poff, L.pcol, L.pval, f4p(W->x[l + 1]), f4m(out));
    OB_CHECK_LAUNCH("amg prolong");
    // Post-smoothing: out -> other -> out.
    sweep_kernel<false><<<grid, kThreads, 0, stream>>>(L.n, G, L.off, L.col, L.val, L.damped, f4p(b),
                                                        f4p(out), f4m(other), nullptr, nullptr, nullptr);
    OB_CHECK_LAUNCH("amg sweep");
    if (top_dot)
        sweep_kernel<true><<<W->blocks, kThreads, smem, stream>>>(L.n, G, L.off, L.col, L.val, L.damped, f4p(b),
                                                                  f4p(other), f4m(out), W->partials,
                                                                  W->counters + 0, W->cols);
    else
        sweep_kernel<false><<<grid, kThreads, 0, stream>>>(L.n, G, L.off, L.col, L.val, L.damped, f4p(b),
                                                            f4p(other), f4m(out), nullptr, nullptr, nullptr);
    OB_CHECK_LAUNCH("amg sweep");
    *launches += 3;
    return OB_OK;
}

// One inner CG iteration (the loop body before its decision).
int enqueue_iteration(Amg* M, Work* W, cudaStream_t stream, int* launches) {
    const int G = W->G;
    const size_t smem = partial_smem(G);
    const DeviceLevel& L = M->levels[0];
    auto f4p = [](const float* p) { return reinterpret_cast<const float4*>(p); };
    auto f4m = [](float* p) { return reinterpret_cast<float4*>(p); };
    direction_kernel<<<W->blocks, kThreads, smem, stream>>>(M->n, G, L.off, L.col, L.val, f4p(W->z), f4m(W->p),
                                                            f4m(W->q), W->partials, W->counters + 1, W->cols);
    OB_CHECK_LAUNCH("amg direction");
    update_kernel<<<W->blocks, kThreads, smem, stream>>>(M->n, G, f4p(W->p), f4p(W->q), f4m(W->d), f4m(W->res),
                                                         W->partials, W->counters + 2, W->cols, W->loop);
    OB_CHECK_LAUNCH("amg update");
    *launches += 2;
    return enqueue_cycle(M, W, 0, W->res, W->z, true, stream, launches);
}

int inner_graph(Amg* M, Work* W) {
    if (W->inner) return OB_OK;
    if (!M->capture) OB_CUDA(cudaStreamCreateWithFlags(&M->capture, cudaStreamNonBlocking));
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
    e = cudaStreamBeginCaptureToGraph(M->capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_status(e, "cudaStreamBeginCaptureToGraph");
    }
    suppress_counting(1);
    int launches = 0;
    int st = enqueue_iteration(M, W, M->capture, &launches);
    if (st == OB_OK) {
        decide_kernel<<<1, 128, 0, M->capture>>>(W->cols, W->kp, W->loop, handle);
        ++launches;
    }
    suppress_counting(-1);
    cudaGraph_t captured;
    e = cudaStreamEndCapture(M->capture, &captured);
    if (st != OB_OK || e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return st != OB_OK ? st : cuda_status(e, "cudaStreamEndCapture(amg)");
    }
    cudaGraphExec_t exec;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return cuda_status(e, "cudaGraphInstantiate(amg)");
    }
    W->inner_graph = graph;
    W->inner = exec;
    W->inner_launches = launches;
    return OB_OK;
}

int check_columns(int k, int ld) {
    if (k < 1) return fail(OB_ERR_INVALID, "amg: k must be >= 1");
    if (ld < k) return fail(OB_ERR_INVALID, "amg: ld must be >= k");
    return OB_OK;
}

}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

// The hierarchy of a large operator: its levels of at least kDeviceLevelRows rows built on the
// device (build_device_levels), the rest on the host from the level the device handed over.
// Where the large levels of a hierarchy are built (ob_amg_build_mode): 1 the device (default),
// 0 the host (the comparison of the two).
std::atomic<int> g_build_on_device{1};
bool amg_build_on_device() { return g_build_on_device.load() != 0; }

int setup_on_device(Amg* M, int n, long long nnz, const int32_t* offsets, const int32_t* columns,
                    const double* values, unsigned seed, cudaStream_t stream) {
    DevBuild B;
    int st = build_device_levels(DevCsr{n, n, nnz, offsets, columns, values}, seed, kDeviceLevelRows, &B, stream);
    // Whatever the build kept is the handle's from here (released with it).
    M->allocations.insert(M->allocations.end(), B.owned.begin(), B.owned.end());
    B.owned.clear();
    if (st) return st;
    void* p = nullptr;
    OB_CUDA(cudaMalloc(&p, sizeof(float) * (size_t)n));
    M->allocations.push_back(p);
    M->jacobi = static_cast<float*>(p);
    dev_jacobi_kernel<<<grid_of(n), kThreads, 0, stream>>>(n, offsets, columns, values, M->jacobi);
    OB_CHECK_LAUNCH("amg jacobi");
    // The host's part, from the last device level on.
    const int device_levels = (int)B.levels.size() - 1;
    HCsr handover = download(B.levels.back().A, stream, &st);
    if (st) return st;
    HostHierarchy H;
    build_hierarchy_from(std::move(handover), seed, B.weights, device_levels, !B.stopped, &H);
    M->usable = H.usable;
    if (!H.usable) {
        // The Jacobi preconditioner in its place: level 0 only, as the host build leaves it.
        M->levels.resize(1);
        DeviceLevel& d = M->levels[0];
        d.n = n;
        d.nnz = nnz;
        d.off = const_cast<int*>(offsets);
        d.col = const_cast<int*>(columns);
        OB_CUDA(cudaMalloc(&p, sizeof(float) * (size_t)std::max(nnz, 1LL)));
        M->allocations.push_back(p);
        d.val = static_cast<float*>(p);
        dev_narrow_kernel<<<grid_of(nnz), kThreads, 0, stream>>>(nnz, values, d.val);
        OB_CHECK_LAUNCH("amg narrow");
        OB_CUDA(cudaStreamSynchronize(stream));
        return OB_OK;
    }
    M->levels.resize((size_t)device_levels + H.levels.size());
    auto narrow_to = [&](const double* in, long long count, float** out) -> int {
        void* q = nullptr;
        OB_CUDA(cudaMalloc(&q, sizeof(float) * (size_t)std::max(count, 1LL)));
        M->allocations.push_back(q);
        *out = static_cast<float*>(q);
        if (count > 0) {
            dev_narrow_kernel<<<grid_of(count), kThreads, 0, stream>>>(count, in, *out);
            OB_CHECK_LAUNCH("amg narrow");
        }
        return OB_OK;
    };
    for (int l = 0; l < device_levels && st == OB_OK; ++l) {
        const DevLevel& g = B.levels[l];
        DeviceLevel& d = M->levels[l];
        d.n = g.A.rows;
        d.nnz = g.A.nnz;
        d.off = const_cast<int*>(g.A.off);
        d.col = const_cast<int*>(g.A.col);
        d.n_coarse = g.P.cols;
        d.pnnz = g.P.nnz;
        d.rnnz = g.R.nnz;
        d.poff = const_cast<int*>(g.P.off);
        d.pcol = const_cast<int*>(g.P.col);
        d.roff = const_cast<int*>(g.R.off);
        d.rcol = const_cast<int*>(g.R.col);
        if ((st = narrow_to(g.A.val, g.A.nnz, &d.val)) || (st = narrow_to(g.damped, g.A.rows, &d.damped)) ||
            (st = narrow_to(g.P.val, g.P.nnz, &d.pval)) || (st = narrow_to(g.R.val, g.R.nnz, &d.rval)))
            break;
    }
    for (size_t h = 0; h < H.levels.size() && st == OB_OK; ++h) {
        HostLevel& hl = H.levels[h];
        DeviceLevel& d = M->levels[(size_t)device_levels + h];
        d.n = hl.A.rows;
        d.nnz = hl.A.nnz();
        if ((st = upload(M, hl.A.off, &d.off, stream)) || (st = upload(M, hl.A.col, &d.col, stream)) ||
            (st = upload(M, narrow(hl.A.val), &d.val, stream)))
            break;
        if (!hl.damped.empty()) {
            d.n_coarse = hl.P.cols;
            d.pnnz = hl.P.nnz();
            d.rnnz = hl.R.nnz();
            if ((st = upload(M, narrow(hl.damped), &d.damped, stream)) || (st = upload(M, hl.P.off, &d.poff, stream)) ||
                (st = upload(M, hl.P.col, &d.pcol, stream)) || (st = upload(M, narrow(hl.P.val), &d.pval, stream)) ||
                (st = upload(M, hl.R.off, &d.roff, stream)) || (st = upload(M, hl.R.col, &d.rcol, stream)) ||
                (st = upload(M, narrow(hl.R.val), &d.rval, stream)))
                break;
        }
    }
    if (st) return st;
    const int rows = H.levels.back().A.rows;
    M->coarse_rows = rows;
    M->n_active = (int)H.active.size();
    std::vector<int> slots(rows + std::max<size_t>(H.active.size(), 1), -1);
    for (size_t t = 0; t < H.active.size(); ++t) {
        slots[H.active[t]] = (int)t;
        slots[rows + t] = H.active[t];
    }
    if ((st = upload(M, slots, &M->slots, stream))) return st;
    if ((st = upload(M, narrow(H.inverse.empty() ? std::vector<double>(1, 0.0) : H.inverse), &M->inverse, stream)))
        return st;
    OB_CUDA(cudaStreamSynchronize(stream));
    return OB_OK;
}

int ob_amg_setup(int n, const int32_t* offsets, const int32_t* columns, const double* values, unsigned seed,
                 void** amg, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(n >= 1 && offsets && columns && values && amg, "ob_amg_setup: bad argument");
    *amg = nullptr;
    if (n >= kDeviceLevelRows && amg_build_on_device()) {
        int nnz_host = 0;
        OB_CUDA(cudaMemcpyAsync(&nnz_host, offsets + n, sizeof(int), cudaMemcpyDeviceToHost, stream));
        OB_CUDA(cudaStreamSynchronize(stream));
        OB_REQUIRE(nnz_host >= 0, "ob_amg_setup: bad offsets");
        auto M = std::make_unique<Amg>();
        M->n = n;
        M->nnz = nnz_host;
        M->off64 = offsets;
        M->col64 = columns;
        M->val64 = values;
        int st = setup_on_device(M.get(), n, nnz_host, offsets, columns, values, seed, stream);
        if (st) {
            cudaStreamSynchronize(stream);
            release(M.get());
            return st;
        }
        *amg = M.release();
        return OB_OK;
    }
    HCsr fine;
    fine.rows = fine.cols = n;
    fine.off.resize(n + 1);
    OB_CUDA(cudaMemcpyAsync(fine.off.data(), offsets, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, stream));
    OB_CUDA(cudaStreamSynchronize(stream));
    const long long nnz = fine.off[n];
    OB_REQUIRE(nnz >= 0 && fine.off[0] == 0, "ob_amg_setup: bad offsets");
    fine.col.resize(nnz);
    fine.val.resize(nnz);
    if (nnz) {
        OB_CUDA(cudaMemcpyAsync(fine.col.data(), columns, sizeof(int) * nnz, cudaMemcpyDeviceToHost, stream));
        OB_CUDA(cudaMemcpyAsync(fine.val.data(), values, sizeof(double) * nnz, cudaMemcpyDeviceToHost, stream));
        OB_CUDA(cudaStreamSynchronize(stream));
    }
    for (long long e = 0; e < nnz; ++e)
        if (fine.col[e] < 0 || fine.col[e] >= n) return fail(OB_ERR_INDEX, "ob_amg_setup: column out of range");
    auto M = std::make_unique<Amg>();
    M->n = n;
    M->nnz = nnz;
    M->off64 = offsets;
    M->col64 = columns;
    M->val64 = values;
    HostHierarchy H;
    build_hierarchy(std::move(fine), seed, &H);
    int st = OB_OK;
    M->usable = H.usable;
    st = upload(M.get(), narrow(H.jacobi), &M->jacobi, stream);
    const size_t levels = H.usable ? H.levels.size() : 1;
    M->levels.resize(levels);
    for (size_t l = 0; l < levels && st == OB_OK; ++l) {
        HostLevel& h = H.levels[l];
        DeviceLevel& d = M->levels[l];
        d.n = h.A.rows;
        d.nnz = h.A.nnz();
        if ((st = upload(M.get(), h.A.off, &d.off, stream))) break;
        if ((st = upload(M.get(), h.A.col, &d.col, stream))) break;
        if ((st = upload(M.get(), narrow(h.A.val), &d.val, stream))) break;
        if (!h.damped.empty()) {
            d.n_coarse = h.P.cols;
            d.pnnz = h.P.nnz();
            d.rnnz = h.R.nnz();
            if ((st = upload(M.get(), narrow(h.damped), &d.damped, stream))) break;
            if ((st = upload(M.get(), h.P.off, &d.poff, stream))) break;
            if ((st = upload(M.get(), h.P.col, &d.pcol, stream))) break;
            if ((st = upload(M.get(), narrow(h.P.val), &d.pval, stream))) break;
            if ((st = upload(M.get(), h.R.off, &d.roff, stream))) break;
            if ((st = upload(M.get(), h.R.col, &d.rcol, stream))) break;
            if ((st = upload(M.get(), narrow(h.R.val), &d.rval, stream))) break;
        }
    }
    if (st == OB_OK && H.usable) {
        const int rows = H.levels.back().A.rows;
        M->coarse_rows = rows;
        M->n_active = (int)H.active.size();
        std::vector<int> slots(rows + std::max<size_t>(H.active.size(), 1), -1);
        for (size_t t = 0; t < H.active.size(); ++t) {
            slots[H.active[t]] = (int)t;
            slots[rows + t] = H.active[t];
        }
        st = upload(M.get(), slots, &M->slots, stream);
        if (st == OB_OK) st = upload(M.get(), narrow(H.inverse.empty() ? std::vector<double>(1, 0.0) : H.inverse),
                                     &M->inverse, stream);
    }
    if (st == OB_OK) {
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) st = cuda_status(e, "ob_amg_setup");
    }
    if (st) {
        release(M.get());
        return st;
    }
    *amg = M.release();
    return OB_OK;
}

int ob_amg_build_mode(int on_device) {
    g_build_on_device.store(on_device != 0);
    return OB_OK;
}

int ob_amg_destroy(void* amg) {
    if (!amg) return OB_OK;
    Amg* M = static_cast<Amg*>(amg);
    release(M);
    delete M;
    return OB_OK;
}

int ob_amg_info(void* amg, long long* info) {
    OB_REQUIRE(amg && info, "ob_amg_info: bad argument");
    Amg* M = static_cast<Amg*>(amg);
    info[0] = M->usable ? (long long)M->levels.size() : 0;
    info[1] = M->usable ? M->coarse_rows : 0;
    info[2] = M->n_active;
    long long nnz = 0;
    for (auto& L : M->levels) nnz += L.nnz;
    info[3] = nnz;
    return OB_OK;
}

int ob_amg_levels(void* amg, long long* rows, long long* nnz, int capacity) {
    OB_REQUIRE(amg && rows && nnz && capacity >= 1, "ob_amg_levels: bad argument");
    Amg* M = static_cast<Amg*>(amg);
    const int count = std::min<int>(capacity, (int)M->levels.size());
    for (int l = 0; l < count; ++l) {
        rows[l] = M->levels[l].n;
        nnz[l] = M->levels[l].nnz;
    }
    return OB_OK;
}

int ob_amg_time_kernels(void* amg, int k, int reps, float* ms, long long* bytes, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(amg && ms && bytes && reps >= 1 && k >= 1 && k <= kMaxColumns, "ob_amg_time_kernels: bad argument");
    Amg* M = static_cast<Amg*>(amg);
    OB_REQUIRE(M->usable && M->levels.size() >= 2, "ob_amg_time_kernels: no multigrid hierarchy");
    std::lock_guard<std::mutex> guard(M->lock);
    const int kp = padded_columns(k);
    Work* W;
    int st = ensure_work(M, kp, &W, stream);
    if (st) return st;
    const DeviceLevel& L = M->levels[0];
    const DeviceLevel& C = M->levels[1];
    const size_t vec = sizeof(float) * (size_t)L.n * kp, coarse = sizeof(float) * (size_t)C.n * kp;
    // Defined inputs (zeros) for every vector the timed kernels read.
    OB_CUDA(cudaMemsetAsync(W->res, 0, vec, stream));
    OB_CUDA(cudaMemsetAsync(W->y[0], 0, vec, stream));
    OB_CUDA(cudaMemsetAsync(W->z, 0, vec, stream));
    OB_CUDA(cudaMemsetAsync(W->r[0], 0, vec, stream));
    OB_CUDA(cudaMemsetAsync(W->x[1], 0, coarse, stream));
    const int G = W->G;
    const int grid = grid_for((long long)L.n * G), coarse_grid = grid_for((long long)C.n * G);
    auto f4p = [](const float* p) { return reinterpret_cast<const float4*>(p); };
    auto f4m = [](float* p) { return reinterpret_cast<float4*>(p); };
    const long long matrix = 4LL * (L.n + 1) + 8LL * L.nnz;
    // Algorithmic bytes: each stored entry (column + value) and offset once, every vector row once.
    bytes[0] = matrix + 4LL * L.n + 3LL * (long long)vec;                             // sweep
    bytes[1] = matrix + 3LL * (long long)vec;                                         // residual
    bytes[2] = 4LL * (C.n + 1) + 8LL * L.rnnz + (long long)vec + (long long)coarse;   // restriction
    bytes[3] = 4LL * (L.n + 1) + 8LL * L.pnnz + (long long)coarse + 2LL * (long long)vec;  // prolongation
    bytes[4] = 0;                                                                     // whole V-cycle
    cudaEvent_t marks[6];
    for (auto& e : marks) OB_CUDA(cudaEventCreate(&e));
    auto kernel = [&](int which) {
        switch (which) {
            case 0:
                sweep_kernel<false><<<grid, kThreads, 0, stream>>>(L.n, G, L.off, L.col, L.val, L.damped, f4p(W->res),
                                                                    f4p(W->y[0]), f4m(W->z), nullptr, nullptr,
                                                                    nullptr);
                break;
            case 1:
                residual_kernel<<<grid, kThreads, 0, stream>>>(L.n, G, L.off, L.col, L.val, f4p(W->res),
                                                               f4p(W->z), f4m(W->r[0]));
                break;
            case 2:
                spmm_kernel<false><<<coarse_grid, kThreads, 0, stream>>>(C.n, G, L.roff, L.rcol, L.rval,
                                                                         f4p(W->r[0]), f4m(W->b[1]));
                break;
            case 3:
                spmm_kernel<true><<<grid, kThreads, 0, stream>>>(L.n, G, L.poff, L.pcol, L.pval, f4p(W->x[1]),
                                                                 f4m(W->z));
                break;
            default: {
                int launches = 0;
                return enqueue_cycle(M, W, 0, W->res, W->z, false, stream, &launches);
            }
        }
        count_launch();
        return cudaGetLastError() == cudaSuccess ? OB_OK : fail(OB_ERR_CUDA, "ob_amg_time_kernels: launch");
    };
    for (int which = 0; which < 5 && st == OB_OK; ++which) st = kernel(which);  // warm-up
    for (int which = 0; which < 5 && st == OB_OK; ++which) {
        cudaEventRecord(marks[which], stream);
        for (int i = 0; i < reps && st == OB_OK; ++i) st = kernel(which);
    }
    cudaEventRecord(marks[5], stream);
    cudaError_t e = cudaEventSynchronize(marks[5]);
    for (int which = 0; which < 5 && e == cudaSuccess; ++which) {
        float total = 0.0f;
        e = cudaEventElapsedTime(&total, marks[which], marks[which + 1]);
        ms[which] = total / (float)reps;
    }
    for (auto& m : marks) cudaEventDestroy(m);
    if (st) return st;
    if (e != cudaSuccess) return cuda_status(e, "ob_amg_time_kernels");
    return OB_OK;
}

int ob_amg_apply(void* amg, const double* b, double* x, int k, int ld, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(amg && b && x, "ob_amg_apply: bad argument");
    Amg* M = static_cast<Amg*>(amg);
    int st = check_columns(k, ld);
    if (st) return st;
    std::lock_guard<std::mutex> guard(M->lock);
    for (int c0 = 0; c0 < k; c0 += kMaxColumns) {
        const int kc = std::min(kMaxColumns, k - c0);
        const int kp = padded_columns(kc);
        Work* W;
        if ((st = ensure_work(M, kp, &W, stream))) return st;
        const int grid = grid_for((long long)M->n * kp);
        to_f32_kernel<<<grid, kThreads, 0, stream>>>(M->n, kc, kp, b + c0, ld, W->res);
        OB_CHECK_LAUNCH("amg to_f32");
        int launches = 0;
        if ((st = enqueue_cycle(M, W, 0, W->res, W->z, false, stream, &launches))) return st;
        from_f32_kernel<<<grid, kThreads, 0, stream>>>(M->n, kc, kp, W->z, x + c0, ld);
        OB_CHECK_LAUNCH("amg from_f32");
    }
    return OB_OK;
}

int ob_amg_solve(void* amg, const double* b, double* x, int k, int ld, double tol, int max_outer,
                 int max_inner, double inner_tol, int* iterations, double* residuals, int* statuses,
                 ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(amg && b && x, "ob_amg_solve: bad argument");
    OB_REQUIRE(tol >= 0.0 && max_outer >= 0 && max_inner >= 1 && inner_tol > 0.0 && inner_tol < 1.0,
               "ob_amg_solve: bad tolerance or iteration caps");
    Amg* M = static_cast<Amg*>(amg);
    int st = check_columns(k, ld);
    if (st) return st;
    std::lock_guard<std::mutex> guard(M->lock);
    for (int c0 = 0; c0 < k; c0 += kMaxColumns) {
        const int kc = std::min(kMaxColumns, k - c0);
        const int kp = padded_columns(kc);
        Work* W;
        if ((st = ensure_work(M, kp, &W, stream))) return st;
        if ((st = inner_graph(M, W))) return st;
        const int G = W->G;
        const size_t smem = partial_smem(G);
        const int grid = grid_for((long long)M->n * kp);
        double* r64 = W->r64;
        gather_columns_kernel<<<grid, kThreads, 0, stream>>>(M->n, kc, kp, b + c0, ld, W->b64);
        OB_CHECK_LAUNCH("amg gather b");
        gather_columns_kernel<<<grid, kThreads, 0, stream>>>(M->n, kc, kp, x + c0, ld, W->x64);
        OB_CHECK_LAUNCH("amg gather x");
        start_kernel<<<W->blocks, kThreads, smem, stream>>>(M->n, G, kc, W->b64, W->partials, W->counters + 3,
                                                            W->cols);
        OB_CHECK_LAUNCH("amg start");
        LoopState loop_host = {0, max_inner, 1, 0, inner_tol * inner_tol};
        for (int outer = 0;; ++outer) {
            refine_residual_kernel<<<W->blocks, kThreads, smem, stream>>>(
                M->n, G, M->off64, M->col64, M->val64, W->b64, W->x64, r64, W->partials, W->counters + 4, W->cols,
                tol * tol);
            OB_CHECK_LAUNCH("amg refine residual");
            OB_CUDA(cudaMemcpyAsync(W->host_cols, W->cols, sizeof(ColumnState) * kp, cudaMemcpyDeviceToHost, stream));
            OB_CUDA(cudaStreamSynchronize(stream));
            bool any = false;
            for (int c = 0; c < kc; ++c) any |= W->host_cols[c].outer_done == 0;
            if (!any || outer >= max_outer) break;
            narrow_kernel<<<grid, kThreads, 0, stream>>>(M->n, kp, r64, W->cols, W->res, W->d, W->p, W->q);
            OB_CHECK_LAUNCH("amg narrow");
            int launches = 0;
            if ((st = enqueue_cycle(M, W, 0, W->res, W->z, true, stream, &launches))) return st;
            OB_CUDA(cudaMemcpyAsync(W->loop, &loop_host, sizeof(LoopState), cudaMemcpyHostToDevice, stream));
            OB_CUDA(cudaGraphLaunch(W->inner, stream));
            LoopState after = {};
            OB_CUDA(cudaMemcpyAsync(&after, W->loop, sizeof(LoopState), cudaMemcpyDeviceToHost, stream));
            correct_kernel<<<grid, kThreads, 0, stream>>>(M->n, kp, W->d, W->cols, W->x64);
            OB_CHECK_LAUNCH("amg correct");
            OB_CUDA(cudaStreamSynchronize(stream));
            count_launch((uint64_t)after.iter * W->inner_launches);
        }
        scatter_columns_kernel<<<grid, kThreads, 0, stream>>>(M->n, kc, kp, W->x64, x + c0, ld);
        OB_CHECK_LAUNCH("amg scatter x");
        OB_CUDA(cudaStreamSynchronize(stream));
        for (int c = 0; c < kc; ++c) {
            const ColumnState& C = W->host_cols[c];
            if (iterations) iterations[c0 + c] = C.iters;
            if (residuals)
                residuals[c0 + c] = C.bnorm2 > 0.0 ? std::sqrt(C.res2 / C.bnorm2) : std::sqrt(C.res2);
            if (statuses) statuses[c0 + c] = C.bnorm2 == 0.0 && C.res2 == 0.0 ? OB_STATUS_CONVERGED : C.status;
        }
    }
    return OB_OK;
}

int ob_amg_host_setup(int n, const int32_t* offsets, const int32_t* columns, const double* values,
                      unsigned seed, long long* rows, long long* nnz, int capacity, int* levels) {
    OB_REQUIRE(n >= 1 && offsets && columns && values && rows && nnz && levels && capacity >= 1,
               "ob_amg_host_setup: bad argument");
    HCsr fine;
    fine.rows = fine.cols = n;
    fine.off.assign(offsets, offsets + n + 1);
    fine.col.assign(columns, columns + offsets[n]);
    fine.val.assign(values, values + offsets[n]);
    HostHierarchy H;
    build_hierarchy(std::move(fine), seed, &H);
    *levels = H.usable ? (int)H.levels.size() : 0;
    for (int l = 0; l < std::min<int>(capacity, (int)H.levels.size()); ++l) {
        rows[l] = H.levels[l].A.rows;
        nnz[l] = H.levels[l].A.nnz();
    }
    return OB_OK;
}

}  // extern "C"
