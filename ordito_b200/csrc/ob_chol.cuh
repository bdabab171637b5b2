// Shared internals of the sparse Cholesky (ob_cholesky.cu: ordering, analysis, solves;
// ob_chol_factor.cu: the numeric factorisation on the device).
#pragma once

#include <memory>
#include <mutex>
#include <vector>

#include "ob_internal.cuh"

namespace ob {

// A supernode of the nested-dissection tree (after level amalgamation).
struct CholNode {
    int start = 0, count = 0;          // own columns [start, start + count) in the new numbering
    int parent = -1;
    std::vector<int> children;
    std::vector<int> off_rows;         // ascending, > start + count - 1
    int level = 0;                     // height from the leaves (leaf = 0)
};

struct FactorPlan;  // the device tables of the numeric factorisation (ob_chol_factor.cu)
void release_plan(FactorPlan* plan);

struct CholAnalysis {
    int n = 0;
    std::vector<int> perm;   // new -> old
    std::vector<int> iperm;  // old -> new
    std::vector<int> offsets, columns;  // the operator's pattern (old numbering)
    std::vector<CholNode> nodes;        // postorder: children before parents
    std::vector<int> component_last;    // per vertex (old): is it its component's pin (1/0)
    std::vector<int> component;         // per vertex (old): its connected component, 0 ..
    int n_components = 0;
    long long factor_entries = 0;       // sum of nc * nc + (m - nc) * nc
    int levels = 0;
    // Built on the first numeric factorisation on the device and kept with the analysis (every
    // operator of this pattern shares it: the heat and the Poisson systems).
    std::mutex plan_mutex;
    FactorPlan* plan = nullptr;
    ~CholAnalysis() { release_plan(plan); }
};

// Where each supernode's block [L11^-1; G] (nc + noff rows of ld = nc rounded up to 8 doubles)
// starts in the factor's value buffer, and where its row lists start in the index buffer.
struct BlockLayout {
    std::vector<long long> inv_at, off_at;
    std::vector<int> rows_at, back_at, ld_at;
    long long total = 0, total_rows = 0;
};

inline BlockLayout block_layout(const CholAnalysis& A) {
    BlockLayout B;
    const int ns = (int)A.nodes.size();
    B.inv_at.resize(ns);
    B.off_at.resize(ns);
    B.rows_at.resize(ns);
    B.back_at.resize(ns);
    B.ld_at.resize(ns);
    for (int s = 0; s < ns; ++s) {
        const int nc = A.nodes[s].count, noff = (int)A.nodes[s].off_rows.size();
        const int ld = (nc + 7) / 8 * 8;
        B.ld_at[s] = ld;
        B.inv_at[s] = B.total;
        B.total += (long long)nc * ld;
        B.off_at[s] = B.total;
        B.total += (long long)noff * ld;
        B.rows_at[s] = (int)B.total_rows;
        B.total_rows += noff;
        B.back_at[s] = (int)B.total_rows;
        B.total_rows += nc + noff;
    }
    return B;
}

// Singular-component handling of a numeric factorisation: kPinNone factors the operator as it is;
// kPinAll pins the last vertex (in the new numbering) of every connected component; kPinZeroSum
// pins it only on components whose rows all sum to zero (|row sum| <= 1e-10 |diagonal|, the
// reference's test of a Laplacian's constant null space, ordito/cholesky.py:76).
enum PinMode : int { kPinNone = 0, kPinAll = 1, kPinZeroSum = 2 };

// Numeric factorisation of sign * values (CSR over the analysis' pattern, old numbering) on the
// device, multifrontal over the tree, level by level: writes every supernode's [L11^-1; G] block
// into vals (laid out by block_layout, zeroed here) and pinned[n] (new numbering). Returns
// OB_ERR_INDEFINITE on a non-positive pivot (read back once at the end).
int device_factor(CholAnalysis& A, const double* values, double sign, int pin_mode, double* vals,
                  char* pinned, cudaStream_t stream);

// D (8 x 8) += A (8 x 4) B (4 x 8) in float64 on the tensor cores (mma.sync m8n8k4 .f64, the
// float64 matrix instruction sm_100 offers). Fragments: a = A[lane / 4][lane % 4],
// b = B[lane % 4][lane / 4], d = D[lane / 4][2 (lane % 4) + {0, 1}].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

}  // namespace ob
