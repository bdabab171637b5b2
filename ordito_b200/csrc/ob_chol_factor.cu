// a11: the numeric sparse Cholesky factorisation on the device.
//
// Follows ordito/cholesky.py:1399 _factor (kernels/cholesky.py:434 factor_panel_tiled, :541
// panel_front_product, :591 update_panel_entries, :772-839 factor_front_panels /
// factor_level_panels): multifrontal over the dissection tree, one tree level at a time, every
// front of a level in the same launches. A front is the dense m x m matrix of a supernode's nc own
// columns and noff off-diagonal rows (m = nc + noff), column-major in one arena: it receives the
// operator's entries of its own columns (scattered once, for every front, before the first level)
// and its children's Schur complements (extend-add, child by child in a fixed order, so every
// front entry is summed in the same order on every run: no atomics). Its own columns are then
// eliminated in panels of 64:
//
//   K1  the panel's diagonal block D (b x b, b <= 64): Cholesky and its inverse D^-1, in shared
//       memory (one CTA a front); D^-1 goes straight into the stored block.
//   K2  the panel below the diagonal, L = F D^-T (in place), and the rows of the panel in the
//       stored block, Z_p = D^-1 Z_p (in place).
//   K3  the trailing update, F[j1:, j1:] -= L L^T (lower tiles), and Z[j1:, :j1] -= L Z_p.
//
// Z is the supernode's stored block [L11^-1; G] with G = -L21 L11^-1 -- the first nc columns of
// the inverse of [L11 0; L21 I], which forward elimination of [I; 0] builds panel by panel
// alongside the factorisation, so the partitioned inverse the solves read (ordito/cholesky.py
// notes: Alvarado, Pothen and Schreiber 1993) costs no separate pass. After the last panel the
// front's trailing block is the Schur complement its parent takes. K2 and K3 are batched float64
// tensor-core products (mma.sync m8n8k4) over 64 x 64 output tiles with an inner dimension of one
// panel; the whole schedule (every level's extend-add ranks, panels and tile lists) depends only
// on the analysis, so it is built once per analysis and kept.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ob_chol.cuh"
#include "ob_host.hpp"
#include "ob_scratch.cuh"

namespace ob {

namespace {

constexpr int kPanel = 64;         // columns eliminated a panel step; tile edge of K2 / K3
constexpr int kDiagThreads = 256;
constexpr int kTileThreads = 128;  // four warps, each a 16-row strip of the 64 x 64 output
constexpr int kSmemLd = kPanel + 1;
constexpr int kTileSmem = 2 * kPanel * kSmemLd * (int)sizeof(double);
constexpr int kExtendThreads = 256;
constexpr int kExtendColumns = 32;  // child columns an extend-add task takes
// A row's entries sum to "zero" below this fraction of its diagonal (ordito/cholesky.py:76).
constexpr double kSingularRowSum = 1e-10;

// Extend-add: the child's Schur complement columns [b0, b1) added into its parent's front.
struct ExtendTask {
    int child, parent, b0, b1;
};

// K1: the diagonal block (b x b) of a panel at front offset f (leading dimension fld), its
// inverse written at z in the factor's values (leading dimension zld).
struct DiagTask {
    long long f, z;
    int fld, zld, b, pad;
};

// K2 / K3: C (rows x cols) = or -= A (rows x inner) B (inner x cols), inner <= 64.
// A(i, kk) at a + i a_rs + kk a_ks, B(kk, c) at b + kk b_ks + c b_cs, C(i, c) at c + i c_rs +
// c c_cs; each offset into the front arena (buffer 0) or the factor's values (buffer 1).
struct ProductTile {
    long long a, b, c;
    int a_rs, a_ks, b_ks, b_cs, c_rs, c_cs;
    int rows, cols, inner;
    unsigned char a_buf, b_buf, c_buf, subtract;
};

enum LaunchKind : int { kExtend = 0, kDiag = 1, kProduct = 2 };

}  // namespace

struct FactorPlan {
    int device = -1;
    long long front_total = 0;  // doubles in the front arena
    long long n_entries = 0;    // CSR entries of the operator
    // Per CSR entry (old numbering): its slot in the fronts (-1: the upper triangle, which the
    // lower one mirrors) and the new indices of its row and column.
    long long* entry_dest = nullptr;
    int2* entry_rc = nullptr;
    long long* diag_dest = nullptr;  // per new row: its diagonal slot in its front
    int* diag_pos = nullptr;         // per old row: the CSR position of its diagonal, or -1
    int* component = nullptr;        // per old row
    char* component_last = nullptr;  // per old row
    int* perm = nullptr;             // new -> old
    int* offsets = nullptr;          // the operator's row offsets (old numbering)
    // Per supernode: front offset, front leading dimension, own columns, off-diagonal rows, and
    // where its off-diagonal rows' positions in its parent's front start in `rel`.
    long long* front_at = nullptr;
    int* fld = nullptr;
    int* nc = nullptr;
    int* noff = nullptr;
    int* rel_at = nullptr;
    int* rel = nullptr;
    struct Launch {
        int kind;
        const void* tasks;
        int count;
    };
    std::vector<Launch> launches;  // the whole numeric schedule, in order
    std::vector<void*> owned;
};

void release_plan(FactorPlan* plan) {
    if (plan == nullptr) return;
    if (!plan->owned.empty()) {
        int current = -1;
        cudaGetDevice(&current);
        if (plan->device >= 0 && plan->device != current) cudaSetDevice(plan->device);
        {
            std::lock_guard<std::recursive_mutex> guard(capture_mutex());
            cudaDeviceSynchronize();
        }
        for (void* p : plan->owned) cudaFree(p);
        if (current >= 0 && plan->device >= 0 && plan->device != current) cudaSetDevice(current);
    }
    delete plan;
}

namespace {

template <typename T>
int upload(FactorPlan* P, T** out, const std::vector<T>& host, cudaStream_t stream) {
    void* p = nullptr;
    OB_CUDA(pool_malloc(&p, sizeof(T) * std::max<size_t>(host.size(), 1), stream));
    P->owned.push_back(p);
    if (!host.empty())
        OB_CUDA(cudaMemcpyAsync(p, host.data(), sizeof(T) * host.size(), cudaMemcpyHostToDevice, stream));
    *out = static_cast<T*>(p);
    return OB_OK;
}

template <typename T>
int allocate(FactorPlan* P, T** out, size_t count, cudaStream_t stream) {
    void* p = nullptr;
    OB_CUDA(pool_malloc(&p, sizeof(T) * std::max<size_t>(count, 1), stream));
    P->owned.push_back(p);
    *out = static_cast<T*>(p);
    return OB_OK;
}

template <typename T>
int upload_scratch(Scratch& scratch, const T** out, const std::vector<T>& host, cudaStream_t stream) {
    T* p = scratch.take<T>(host.size());
    if (int st = scratch.commit()) return st;
    if (!host.empty())
        OB_CUDA(cudaMemcpyAsync(p, host.data(), sizeof(T) * host.size(), cudaMemcpyHostToDevice, stream));
    *out = p;
    return OB_OK;
}

// The tree as the plan kernels read it: per supernode its first column, own columns, front
// offset and leading dimension, and its off-diagonal rows (ascending) at rows + row_at[s] ..
// row_at[s + 1]; per new column its supernode.
struct PlanTree {
    const int* start;
    const int* nc;
    const long long* front_at;
    const int* fld;
    const int* row_at;
    const int* rows;
    const int* node_of;
};

// Row r's position in supernode s's front: its own column r - start, else nc + its index among
// the off-diagonal rows (which hold r: the symbolic structure puts it there).
__device__ __forceinline__ int front_position(const PlanTree& T, int s, int r) {
    const int start = T.start[s], count = T.nc[s];
    if (r < start + count) return r - start;
    int lo = T.row_at[s], hi = T.row_at[s + 1];
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (T.rows[mid] < r) lo = mid + 1;
        else hi = mid;
    }
    return count + (lo - T.row_at[s]);
}

// node_of[j] = s for each own column j of supernode s (a warp a supernode).
__global__ void node_of_kernel(int ns, const int* __restrict__ start, const int* __restrict__ nc, int* node_of) {
    const int s = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    if (s >= ns) return;
    for (int j = threadIdx.x & 31; j < nc[s]; j += 32) node_of[start[s] + j] = s;
}

// Per CSR entry e of old row ro (a group of 8 lanes a row): its new (row, column) and its slot
// in the front of its row's supernode (-1 in the upper triangle, which the lower one mirrors);
// per old row the CSR position of its diagonal (left -1 when it has none).
constexpr int kEntryLanes = 8;
__global__ void entries_kernel(int n, const int* __restrict__ offsets, const int* __restrict__ columns,
                               const int* __restrict__ iperm, const PlanTree T, long long* __restrict__ dest,
                               int2* __restrict__ rc, int* __restrict__ diag_pos) {
    const long long lane_id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int ro = (int)(lane_id / kEntryLanes);
    if (ro >= n) return;
    const int lane = (int)(lane_id % kEntryLanes);
    const int j = iperm[ro];
    const int s = T.node_of[j];
    const long long column_at = T.front_at[s] + (long long)(j - T.start[s]) * T.fld[s];
    for (int e = offsets[ro] + lane; e < offsets[ro + 1]; e += kEntryLanes) {
        const int co = columns[e];
        const int r = iperm[co];
        rc[e] = make_int2(j, r);
        if (co == ro) diag_pos[ro] = e;
        dest[e] = r < j ? -1LL : column_at + front_position(T, s, r);
    }
}

// rel: each child's off-diagonal rows as positions in its parent's front (a warp a supernode;
// a root's entries are left unset: nothing reads them).
__global__ void rel_kernel(int ns, const int* __restrict__ parent, const PlanTree T, int* __restrict__ rel) {
    const int s = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    if (s >= ns || parent[s] < 0) return;
    for (int i = T.row_at[s] + (threadIdx.x & 31); i < T.row_at[s + 1]; i += 32)
        rel[i] = front_position(T, parent[s], T.rows[i]);
}

// Each new column's diagonal slot in its supernode's front.
__global__ void diag_dest_kernel(int n, const PlanTree T, long long* __restrict__ diag_dest) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int s = T.node_of[j];
    const long long lj = j - T.start[s];
    diag_dest[j] = T.front_at[s] + lj * T.fld[s] + lj;
}

// The device tables and the launch schedule of an analysis (once). The per-entry and per-row
// tables are built on the device from the tree; the host builds the launch schedule.
int build_plan(const CholAnalysis& A, FactorPlan* P, cudaStream_t stream) {
    const int n = A.n, ns = (int)A.nodes.size();
    const BlockLayout layout = block_layout(A);
    // Front arena: node s is m x m column-major at front_at[s], leading dimension fld (m rounded
    // up to 8 doubles, so every front column starts on 64 bytes).
    std::vector<long long> front_at(ns);
    std::vector<int> fld(ns), nc(ns), noff(ns), start(ns), parent(ns), row_at(ns + 1, 0);
    long long total = 0;
    for (int s = 0; s < ns; ++s) {
        const CholNode& nd = A.nodes[s];
        nc[s] = nd.count;
        start[s] = nd.start;
        parent[s] = nd.parent;
        noff[s] = (int)nd.off_rows.size();
        row_at[s + 1] = row_at[s] + noff[s];
        const int m = nc[s] + noff[s];
        fld[s] = (m + 7) / 8 * 8;
        front_at[s] = total;
        total += (long long)fld[s] * m;
    }
    P->front_total = total;
    std::vector<int> rows(row_at[ns]);
    parallel_range(ns, row_at[ns] > (1 << 18), [&](long long lo, long long hi) {
        for (long long s = lo; s < hi; ++s)
            std::copy(A.nodes[s].off_rows.begin(), A.nodes[s].off_rows.end(), rows.begin() + row_at[s]);
    });
    std::vector<char> component_last(n);
    for (int i = 0; i < n; ++i) component_last[i] = (char)A.component_last[i];
    const long long nnz = A.offsets[n];
    P->n_entries = nnz;
    int st = OB_OK;
    if ((st = upload(P, &P->component, A.component, stream)) ||
        (st = upload(P, &P->component_last, component_last, stream)) ||
        (st = upload(P, &P->perm, A.perm, stream)) || (st = upload(P, &P->offsets, A.offsets, stream)) ||
        (st = upload(P, &P->front_at, front_at, stream)) ||
        (st = upload(P, &P->fld, fld, stream)) || (st = upload(P, &P->nc, nc, stream)) ||
        (st = upload(P, &P->noff, noff, stream)) || (st = upload(P, &P->rel_at, row_at, stream)) ||
        (st = allocate(P, &P->rel, (size_t)row_at[ns], stream)) ||
        (st = allocate(P, &P->entry_dest, (size_t)nnz, stream)) ||
        (st = allocate(P, &P->entry_rc, (size_t)nnz, stream)) ||
        (st = allocate(P, &P->diag_pos, (size_t)n, stream)) ||
        (st = allocate(P, &P->diag_dest, (size_t)n, stream)))
        return st;
    {
        // The tree and the pattern, for the table kernels only.
        Scratch scratch(stream);
        const int *d_start = nullptr, *d_parent = nullptr, *d_rows = nullptr, *d_iperm = nullptr,
                  *d_columns = nullptr;
        int* d_node_of = scratch.take<int>((size_t)n);
        if ((st = scratch.commit()) || (st = upload_scratch(scratch, &d_start, start, stream)) ||
            (st = upload_scratch(scratch, &d_parent, parent, stream)) ||
            (st = upload_scratch(scratch, &d_rows, rows, stream)) ||
            (st = upload_scratch(scratch, &d_iperm, A.iperm, stream)) ||
            (st = upload_scratch(scratch, &d_columns, A.columns, stream)))
            return st;
        const PlanTree T{d_start, P->nc, P->front_at, P->fld, P->rel_at, d_rows, d_node_of};
        const int threads = 256;
        node_of_kernel<<<ceil_div(32LL * ns, threads), threads, 0, stream>>>(ns, d_start, P->nc, d_node_of);
        OB_CHECK_LAUNCH("chol plan node_of");
        OB_CUDA(cudaMemsetAsync(P->diag_pos, 0xFF, sizeof(int) * (size_t)n, stream));
        entries_kernel<<<ceil_div((long long)kEntryLanes * n, threads), threads, 0, stream>>>(
            n, P->offsets, d_columns, d_iperm, T, P->entry_dest, P->entry_rc, P->diag_pos);
        OB_CHECK_LAUNCH("chol plan entries");
        rel_kernel<<<ceil_div(32LL * ns, threads), threads, 0, stream>>>(ns, d_parent, T, P->rel);
        OB_CHECK_LAUNCH("chol plan rel");
        diag_dest_kernel<<<ceil_div(n, threads), threads, 0, stream>>>(n, T, P->diag_dest);
        OB_CHECK_LAUNCH("chol plan diagonal slots");
        // The scratch is released in stream order, after these kernels.
    }
    // The schedule, level by level.
    std::vector<std::vector<int>> at_level(A.levels);
    for (int s = 0; s < ns; ++s) at_level[A.nodes[s].level].push_back(s);
    std::vector<ExtendTask> extend;
    std::vector<DiagTask> diag;
    std::vector<ProductTile> tiles;
    // Task lists are gathered on the host per launch, then uploaded as one array each.
    struct Pending {
        int kind;
        size_t first, count;
    };
    std::vector<Pending> pending;
    auto add = [&](int kind, size_t first, size_t count) {
        if (count > 0) pending.push_back(Pending{kind, first, count});
    };
    for (int l = 0; l < A.levels; ++l) {
        const std::vector<int>& nodes = at_level[l];
        size_t ranks = 0;
        for (int s : nodes) ranks = std::max(ranks, A.nodes[s].children.size());
        for (size_t rank = 0; rank < ranks; ++rank) {
            const size_t first = extend.size();
            for (int p : nodes) {
                if (A.nodes[p].children.size() <= rank) continue;
                const int c = A.nodes[p].children[rank];
                for (int b0 = 0; b0 < noff[c]; b0 += kExtendColumns)
                    extend.push_back(ExtendTask{c, p, b0, std::min(noff[c], b0 + kExtendColumns)});
            }
            add(kExtend, first, extend.size() - first);
        }
        int steps = 0;
        for (int s : nodes) steps = std::max(steps, (nc[s] + kPanel - 1) / kPanel);
        for (int step = 0; step < steps; ++step) {
            const int j0 = step * kPanel;
            const size_t d_first = diag.size(), k2_first = tiles.size();
            for (int s : nodes) {
                if (nc[s] <= j0) continue;
                const int b = std::min(kPanel, nc[s] - j0), j1 = j0 + b, m = nc[s] + noff[s];
                const long long f = front_at[s];
                const long long z = layout.inv_at[s];
                const int ld = layout.ld_at[s], fl = fld[s];
                diag.push_back(DiagTask{f + (long long)j0 * fl + j0, z + (long long)j0 * ld + j0, fl, ld, b, 0});
                // K2: L = F D^-T for rows [j1, m) (in place), D^-1 from the stored block.
                for (int rb = j1; rb < m; rb += kPanel) {
                    ProductTile t{};
                    t.a = f + (long long)j0 * fl + rb;
                    t.a_rs = 1;
                    t.a_ks = fl;
                    t.b = z + (long long)j0 * ld + j0;  // B(kk, c) = D^-1(c, kk)
                    t.b_ks = 1;
                    t.b_cs = ld;
                    t.c = t.a;
                    t.c_rs = 1;
                    t.c_cs = fl;
                    t.rows = std::min(kPanel, m - rb);
                    t.cols = b;
                    t.inner = b;
                    t.a_buf = 0, t.b_buf = 1, t.c_buf = 0, t.subtract = 0;
                    tiles.push_back(t);
                }
                // K2: the panel's rows of the stored block, Z_p = D^-1 Z_p over columns [0, j0).
                for (int cb = 0; cb < j0; cb += kPanel) {
                    ProductTile t{};
                    t.a = z + (long long)j0 * ld + j0;  // A(i, kk) = D^-1(i, kk)
                    t.a_rs = ld;
                    t.a_ks = 1;
                    t.b = z + (long long)j0 * ld + cb;  // B(kk, c) = Z(j0 + kk, cb + c)
                    t.b_ks = ld;
                    t.b_cs = 1;
                    t.c = t.b;
                    t.c_rs = ld;
                    t.c_cs = 1;
                    t.rows = b;
                    t.cols = std::min(kPanel, j0 - cb);
                    t.inner = b;
                    t.a_buf = 1, t.b_buf = 1, t.c_buf = 1, t.subtract = 0;
                    tiles.push_back(t);
                }
            }
            add(kDiag, d_first, diag.size() - d_first);
            add(kProduct, k2_first, tiles.size() - k2_first);
            const size_t k3_first = tiles.size();
            for (int s : nodes) {
                if (nc[s] <= j0) continue;
                const int b = std::min(kPanel, nc[s] - j0), j1 = j0 + b, m = nc[s] + noff[s];
                const long long f = front_at[s];
                const long long z = layout.inv_at[s];
                const int ld = layout.ld_at[s], fl = fld[s];
                // K3: F[rb, cb] -= L[rb] L[cb]^T over the lower tiles of [j1, m)^2.
                for (int cb = j1; cb < m; cb += kPanel)
                    for (int rb = cb; rb < m; rb += kPanel) {
                        ProductTile t{};
                        t.a = f + (long long)j0 * fl + rb;
                        t.a_rs = 1;
                        t.a_ks = fl;
                        t.b = f + (long long)j0 * fl + cb;  // B(kk, c) = L(cb + c, kk)
                        t.b_ks = fl;
                        t.b_cs = 1;
                        t.c = f + (long long)cb * fl + rb;
                        t.c_rs = 1;
                        t.c_cs = fl;
                        t.rows = std::min(kPanel, m - rb);
                        t.cols = std::min(kPanel, m - cb);
                        t.inner = b;
                        t.a_buf = 0, t.b_buf = 0, t.c_buf = 0, t.subtract = 1;
                        tiles.push_back(t);
                    }
                // K3: Z[rb, cb] -= L[rb] Z_p[:, cb] for rows [j1, m), columns [0, j1).
                for (int rb = j1; rb < m; rb += kPanel)
                    for (int cb = 0; cb < j1; cb += kPanel) {
                        ProductTile t{};
                        t.a = f + (long long)j0 * fl + rb;
                        t.a_rs = 1;
                        t.a_ks = fl;
                        t.b = z + (long long)j0 * ld + cb;
                        t.b_ks = ld;
                        t.b_cs = 1;
                        t.c = z + (long long)rb * ld + cb;
                        t.c_rs = ld;
                        t.c_cs = 1;
                        t.rows = std::min(kPanel, m - rb);
                        t.cols = std::min(kPanel, j1 - cb);
                        t.inner = b;
                        t.a_buf = 0, t.b_buf = 1, t.c_buf = 1, t.subtract = 1;
                        tiles.push_back(t);
                    }
            }
            add(kProduct, k3_first, tiles.size() - k3_first);
        }
    }
    ExtendTask* d_extend = nullptr;
    DiagTask* d_diag = nullptr;
    ProductTile* d_tiles = nullptr;
    if ((st = upload(P, &d_extend, extend, stream)) || (st = upload(P, &d_diag, diag, stream)) ||
        (st = upload(P, &d_tiles, tiles, stream)))
        return st;
    for (const Pending& q : pending) {
        const void* base = q.kind == kExtend ? (const void*)(d_extend + q.first)
                           : q.kind == kDiag ? (const void*)(d_diag + q.first)
                                             : (const void*)(d_tiles + q.first);
        P->launches.push_back(FactorPlan::Launch{q.kind, base, (int)q.count});
    }
    OB_CUDA(cudaStreamSynchronize(stream));  // the host tables go out of scope
    return OB_OK;
}

// Per old row: whether its entries sum to zero (relative to its diagonal); a component with one
// row that does not is not singular (bad[component] = 1).
__global__ void zero_sum_rows_kernel(int n, const int* __restrict__ offsets, const double* __restrict__ values,
                                     const int* __restrict__ diag_pos, const int* __restrict__ component,
                                     int* __restrict__ bad) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    double sum = 0.0;
    for (int e = offsets[r]; e < offsets[r + 1]; ++e) sum += values[e];
    const double d = diag_pos[r] >= 0 ? values[diag_pos[r]] : 0.0;
    if (!(fabs(sum) <= kSingularRowSum * fabs(d))) bad[component[r]] = 1;
}

// Per new row: pinned when its diagonal is missing or zero (an unreferenced vertex), or when it
// is the last row of a component that is pinned (every component, or every singular one). A
// pinned row's front column is the identity's.
__global__ void pin_rows_kernel(int n, const int* __restrict__ perm, const double* __restrict__ values,
                                const int* __restrict__ diag_pos, const int* __restrict__ component,
                                const char* __restrict__ component_last, const int* __restrict__ bad,
                                int mode, const long long* __restrict__ diag_dest, char* __restrict__ pinned,
                                double* __restrict__ fronts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int old = perm[i];
    const double d = diag_pos[old] >= 0 ? values[diag_pos[old]] : 0.0;
    bool pin = d == 0.0;
    if (component_last[old]) {
        if (mode == kPinAll) pin = true;
        if (mode == kPinZeroSum && bad[component[old]] == 0) pin = true;
    }
    pinned[i] = pin ? 1 : 0;
    if (pin) fronts[diag_dest[i]] = 1.0;
}

// The operator's lower-triangle entries into their fronts (rows and columns of pinned rows left
// out), times sign.
__global__ void scatter_entries_kernel(long long nnz, const double* __restrict__ values,
                                       const long long* __restrict__ dest, const int2* __restrict__ rc,
                                       const char* __restrict__ pinned, double sign, double* __restrict__ fronts) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    const long long d = dest[e];
    if (d < 0) return;
    const int2 ij = rc[e];
    if (pinned[ij.x] || pinned[ij.y]) return;
    fronts[d] = sign * values[e];
}

// Extend-add: a warp a child column b, its lanes the rows a >= b of the child's Schur complement
// (contiguous in the child's front), added at the parent's positions rel[a], rel[b].
__global__ void __launch_bounds__(kExtendThreads)
extend_add_kernel(const ExtendTask* __restrict__ tasks, const long long* __restrict__ front_at,
                  const int* __restrict__ fld, const int* __restrict__ nc, const int* __restrict__ noff,
                  const int* __restrict__ rel_at, const int* __restrict__ rel, double* __restrict__ fronts) {
    const ExtendTask t = tasks[blockIdx.x];
    const int cm = noff[t.child], cnc = nc[t.child], cld = fld[t.child], pld = fld[t.parent];
    const double* U = fronts + front_at[t.child];
    double* Pf = fronts + front_at[t.parent];
    const int* r = rel + rel_at[t.child];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int b = t.b0 + warp; b < t.b1; b += kExtendThreads / 32) {
        const double* src = U + (size_t)(cnc + b) * cld + cnc;
        double* dst = Pf + (size_t)r[b] * pld;
        for (int a = b + lane; a < cm; a += 32) dst[r[a]] += src[a];
    }
}

// K1: Cholesky of the panel's diagonal block and its inverse, in shared memory. Column j: the
// pivot's square root, the column below scaled, then the trailing lower triangle and the
// inverse's rows below updated (the inverse by forward elimination of the identity). A pivot
// that is not positive sets *status and is replaced by 1, so the launch completes.
__global__ void __launch_bounds__(kDiagThreads)
diag_block_kernel(const DiagTask* __restrict__ tasks, const double* __restrict__ fronts, double* __restrict__ vals,
                  int* __restrict__ status) {
    extern __shared__ double diag_smem[];
    double(*L)[kSmemLd] = reinterpret_cast<double(*)[kSmemLd]>(diag_smem);
    double(*X)[kSmemLd] = reinterpret_cast<double(*)[kSmemLd]>(diag_smem + kPanel * kSmemLd);
    const DiagTask t = tasks[blockIdx.x];
    const int b = t.b;
    const double* F = fronts + t.f;
    for (int e = threadIdx.x; e < kPanel * kPanel; e += kDiagThreads) {
        const int r = e % kPanel, c = e / kPanel;
        L[r][c] = (r < b && c < b && r >= c) ? F[(size_t)c * t.fld + r] : 0.0;
        X[r][c] = r == c ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int j = 0; j < b; ++j) {
        double d = L[j][j];
        const bool bad = !(d > 0.0);
        if (bad) d = 1.0;
        const double root = sqrt(d), inv = 1.0 / root;
        __syncthreads();  // every thread has read L[j][j]
        if (threadIdx.x == 0) {
            L[j][j] = root;
            if (bad) *status = 1;
        }
        for (int i = j + 1 + threadIdx.x; i < b; i += kDiagThreads) L[i][j] *= inv;
        for (int c = threadIdx.x; c <= j; c += kDiagThreads) X[j][c] *= inv;
        __syncthreads();
        const int rest = b - j - 1;
        for (int e = threadIdx.x; e < rest * rest; e += kDiagThreads) {
            const int i = j + 1 + e / rest, k = j + 1 + e % rest;
            if (k <= i) L[i][k] -= L[i][j] * L[k][j];
        }
        for (int e = threadIdx.x; e < rest * (j + 1); e += kDiagThreads) {
            const int i = j + 1 + e / (j + 1), c = e % (j + 1);
            X[i][c] -= L[i][j] * X[j][c];
        }
        __syncthreads();
    }
    double* Z = vals + t.z;
    for (int e = threadIdx.x; e < b * b; e += kDiagThreads) {
        const int i = e / b, c = e % b;
        if (c <= i) Z[(size_t)i * t.zld + c] = X[i][c];
    }
}

// K2 / K3: one 64 x 64 output tile a CTA. A and B are staged whole in shared memory (zero past
// their extents) before any output is written, so a tile may write the block it reads (the
// in-place products of K2); no two tiles of a launch write the same entries, and none reads
// what another writes.
__global__ void __launch_bounds__(kTileThreads)
front_product_kernel(const ProductTile* __restrict__ tiles, double* fronts, double* vals) {
    extern __shared__ double smem[];
    double* As = smem;                     // As[i * kSmemLd + kk]
    double* Bs = smem + kPanel * kSmemLd;  // Bs[kk * kSmemLd + c]
    const ProductTile t = tiles[blockIdx.x];
    const double* A = (t.a_buf ? vals : fronts) + t.a;
    const double* B = (t.b_buf ? vals : fronts) + t.b;
    double* C = (t.c_buf ? vals : fronts) + t.c;
    const int inner4 = (t.inner + 3) & ~3;
    for (int e = threadIdx.x; e < kPanel * inner4; e += kTileThreads) {
        int i, kk;
        if (t.a_rs == 1) {
            i = e % kPanel;
            kk = e / kPanel;
        } else {
            kk = e % inner4;
            i = e / inner4;
        }
        As[i * kSmemLd + kk] = (i < t.rows && kk < t.inner) ? A[(long long)i * t.a_rs + (long long)kk * t.a_ks] : 0.0;
        int c;
        if (t.b_cs == 1) {
            c = e % kPanel;
            kk = e / kPanel;
        } else {
            kk = e % inner4;
            c = e / inner4;
        }
        Bs[kk * kSmemLd + c] = (c < t.cols && kk < t.inner) ? B[(long long)kk * t.b_ks + (long long)c * t.b_cs] : 0.0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wr = warp * 16, fr = lane >> 2, fk = lane & 3;
    if (wr >= t.rows) return;
    double acc[2][8][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int col_groups = (t.cols + 7) / 8;
    for (int k4 = 0; k4 < inner4; k4 += 4) {
        double a[2], bv[8];
#pragma unroll
        for (int i = 0; i < 2; ++i) a[i] = As[(wr + 8 * i + fr) * kSmemLd + k4 + fk];
#pragma unroll
        for (int j = 0; j < 8; ++j) bv[j] = Bs[(k4 + fk) * kSmemLd + 8 * j + fr];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (j < col_groups) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], bv[j]);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int r = wr + 8 * i + fr;
        if (r >= t.rows) continue;
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = 8 * j + 2 * fk + h;
                if (c >= t.cols) continue;
                double* o = C + (long long)r * t.c_rs + (long long)c * t.c_cs;
                *o = t.subtract ? *o - acc[i][j][h] : acc[i][j][h];
            }
    }
}

int allow_product_memory() {
    static int allowed[64] = {};
    int device = 0;
    OB_CUDA(cudaGetDevice(&device));
    if (device >= 0 && device < 64 && allowed[device]) return OB_OK;
    OB_CUDA(cudaFuncSetAttribute(front_product_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
    OB_CUDA(cudaFuncSetAttribute(diag_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
    if (device >= 0 && device < 64) allowed[device] = 1;
    return OB_OK;
}

}  // namespace

int device_factor(CholAnalysis& A, const double* values, double sign, int pin_mode, double* vals, char* pinned,
                  cudaStream_t stream) {
    if (int st = allow_product_memory()) return st;
    FactorPlan* P = nullptr;
    {
        std::lock_guard<std::mutex> guard(A.plan_mutex);
        int device = 0;
        OB_CUDA(cudaGetDevice(&device));
        if (A.plan != nullptr && A.plan->device != device) {
            release_plan(A.plan);
            A.plan = nullptr;
        }
        if (A.plan == nullptr) {
            FactorPlan* fresh = new FactorPlan();
            fresh->device = device;
            int st = build_plan(A, fresh, stream);
            if (st) {
                release_plan(fresh);
                return st;
            }
            A.plan = fresh;
        }
        P = A.plan;
    }
    const int n = A.n;
    const long long vals_count = block_layout(A).total;
    Scratch scratch(stream);
    double* fronts = scratch.take<double>((size_t)P->front_total);
    int* bad = scratch.take<int>((size_t)std::max(A.n_components, 1));
    int* status = scratch.take<int>(1);
    if (int st = scratch.commit()) return st;
    OB_CUDA(cudaMemsetAsync(fronts, 0, sizeof(double) * (size_t)std::max<long long>(P->front_total, 1), stream));
    OB_CUDA(cudaMemsetAsync(vals, 0, sizeof(double) * (size_t)std::max<long long>(vals_count, 1), stream));
    OB_CUDA(cudaMemsetAsync(bad, 0, sizeof(int) * (size_t)std::max(A.n_components, 1), stream));
    OB_CUDA(cudaMemsetAsync(status, 0, sizeof(int), stream));
    const int threads = 256;
    if (pin_mode == kPinZeroSum) {
        zero_sum_rows_kernel<<<ceil_div(n, threads), threads, 0, stream>>>(n, P->offsets, values, P->diag_pos,
                                                                           P->component, bad);
        OB_CHECK_LAUNCH("chol zero-sum rows");
    }
    pin_rows_kernel<<<ceil_div(n, threads), threads, 0, stream>>>(n, P->perm, values, P->diag_pos, P->component,
                                                                  P->component_last, bad, pin_mode, P->diag_dest,
                                                                  pinned, fronts);
    OB_CHECK_LAUNCH("chol pin rows");
    if (P->n_entries > 0) {
        scatter_entries_kernel<<<ceil_div(P->n_entries, threads), threads, 0, stream>>>(
            P->n_entries, values, P->entry_dest, P->entry_rc, pinned, sign, fronts);
        OB_CHECK_LAUNCH("chol scatter entries");
    }
    for (const FactorPlan::Launch& L : P->launches) {
        switch (L.kind) {
            case kExtend:
                extend_add_kernel<<<L.count, kExtendThreads, 0, stream>>>(
                    static_cast<const ExtendTask*>(L.tasks), P->front_at, P->fld, P->nc, P->noff, P->rel_at, P->rel,
                    fronts);
                OB_CHECK_LAUNCH("chol extend-add");
                break;
            case kDiag:
                diag_block_kernel<<<L.count, kDiagThreads, kTileSmem, stream>>>(static_cast<const DiagTask*>(L.tasks),
                                                                        fronts, vals, status);
                OB_CHECK_LAUNCH("chol diagonal blocks");
                break;
            default:
                front_product_kernel<<<L.count, kTileThreads, kTileSmem, stream>>>(
                    static_cast<const ProductTile*>(L.tasks), fronts, vals);
                OB_CHECK_LAUNCH("chol front products");
        }
    }
    int host_status = 0;
    OB_CUDA(cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, stream));
    OB_CUDA(cudaStreamSynchronize(stream));
    return host_status ? OB_ERR_INDEFINITE : OB_OK;
}

}  // namespace ob
