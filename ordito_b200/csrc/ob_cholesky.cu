// a11: sparse Cholesky of the heat path's systems, solved on the GPU.
//
// Follows the structure of ordito/cholesky.py (SparseCholesky :121, _analyse :881, _factor :1399,
// _Solve :1606, _nested_dissection :2227): a nested-dissection ordering (geometric when vertex
// positions are given), a supernodal factor whose supernodes are the dissection tree's nodes
// (each leaf domain and each separator one dense front), the diagonal blocks stored as their
// inverses (a partitioned inverse, so both triangular solves are products), and a singular
// operator's components pinned at one vertex each (kernels/cholesky.py:196). The analysis and the
// numeric factorisation run on the host (multifrontal, dense fronts); the solves run on the device,
// level by level of the tree, as batched dense products over many right-hand sides at once.
//
// Device layout of a factor: per supernode s with own columns [c0, c0 + nc) (in the factor's
// numbering) and m rows R_s (the nc own rows first, then the off-diagonal rows, ascending):
//   inv[s]  nc x nc row-major, the inverse of the diagonal block L11 (lower triangular);
//   off[s]  (m - nc) x nc row-major, the off-diagonal panel L21;
//   rows[s] the m - nc off-diagonal row indices.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <numeric>
#include <thread>
#include <vector>

#include "ob_chol.cuh"
#include "ob_host.hpp"
#include "ob_internal.cuh"

namespace ob {
namespace {

// Vertices a dissection leaf holds when the caller asks for the default (leaf_size <= 0).
constexpr int kDefaultLeafSize = 96;

using Node = CholNode;
using Analysis = CholAnalysis;

// ------------------------------------------------------------------------------------------
// Ordering: recursive coordinate bisection with one-sided vertex separators.
// ------------------------------------------------------------------------------------------

struct Dissector {
    const std::vector<int>& off;
    const std::vector<int>& col;
    const float* xyz;  // may be null: breadth-first level bisection instead
    int leaf_size;
    // Marks per vertex: a separator search stamps one side's vertices with its own number, so
    // subtrees dissected on different host threads (disjoint vertex sets) never see each other's
    // marks; the breadth-first bisection (no positions) runs on one thread with 1 / 2 marks.
    std::unique_ptr<std::atomic<int>[]> side;
    std::atomic<int> stamps{3};
    std::vector<Node> tree;  // built in postorder
    std::vector<int> order;  // new -> old, filled in postorder

    Dissector(const std::vector<int>& o, const std::vector<int>& c, const float* p, int n, int leaf)
        : off(o), col(c), xyz(p), leaf_size(leaf), side(new std::atomic<int>[std::max(n, 1)]) {
        for (int v = 0; v < n; ++v) side[v].store(0, std::memory_order_relaxed);
    }

    int mark(int v) const { return side[v].load(std::memory_order_relaxed); }
    void set(int v, int value) { side[v].store(value, std::memory_order_relaxed); }

    // Splits `verts` into (a, b) halves: by the median of the widest coordinate, or by BFS levels.
    void bisect(std::vector<int>& verts, std::vector<int>& a, std::vector<int>& b) {
        const size_t half = verts.size() / 2;
        if (xyz != nullptr) {
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int v : verts)
                for (int d = 0; d < 3; ++d) {
                    lo[d] = std::min(lo[d], xyz[3 * v + d]);
                    hi[d] = std::max(hi[d], xyz[3 * v + d]);
                }
            int axis = 0;
            for (int d = 1; d < 3; ++d)
                if (hi[d] - lo[d] > hi[axis] - lo[axis]) axis = d;
            auto key = [&](int v) { return std::make_pair(xyz[3 * v + axis], v); };
            std::nth_element(verts.begin(), verts.begin() + half, verts.end(),
                             [&](int x, int y) { return key(x) < key(y); });
        } else {
            // Breadth-first order from the first vertex; the first half of the visit is `a`.
            for (int v : verts) set(v, 1);
            std::vector<int> queue;
            queue.reserve(verts.size());
            std::vector<int> visited;
            for (int seed : verts) {
                if (mark(seed) != 1) continue;
                set(seed, 2);
                queue.push_back(seed);
                for (size_t h = visited.size(); h < queue.size(); ++h) {
                    const int v = queue[h];
                    for (int e = off[v]; e < off[v + 1]; ++e)
                        if (mark(col[e]) == 1) {
                            set(col[e], 2);
                            queue.push_back(col[e]);
                        }
                }
                visited = queue;
            }
            for (int v : verts) set(v, 0);
            verts = queue;
        }
        a.assign(verts.begin(), verts.begin() + half);
        b.assign(verts.begin() + half, verts.end());
    }

    // Subtrees of at least this many vertices, down to this depth, are dissected on a thread of
    // their own (geometric bisection only); the tree and the ordering are the same as one
    // thread's: each subtree is built into its own lists and appended in postorder.
    static constexpr int kParallelDepth = 5;
    static constexpr size_t kParallelVertices = 8192;

    // Builds the subtree of `verts` into `tree` / `order` (postorder, indices within the lists);
    // returns its root's index.
    int dissect(std::vector<int> verts, std::vector<Node>& tree_out, std::vector<int>& order_out, int depth) {
        if ((int)verts.size() <= leaf_size) {
            std::sort(verts.begin(), verts.end());
            Node leaf;
            leaf.start = (int)order_out.size();
            leaf.count = (int)verts.size();
            order_out.insert(order_out.end(), verts.begin(), verts.end());
            tree_out.push_back(leaf);
            return (int)tree_out.size() - 1;
        }
        std::vector<int> a, b;
        bisect(verts, a, b);
        // One-sided separator: the vertices of the smaller-boundary side adjacent to the other.
        const int stamp = stamps.fetch_add(1);
        for (int v : b) set(v, stamp);
        std::vector<int> sep, rest_a;
        for (int v : a) {
            bool cut = false;
            for (int e = off[v]; e < off[v + 1] && !cut; ++e) cut = mark(col[e]) == stamp;
            (cut ? sep : rest_a).push_back(v);
        }
        std::vector<int> children;
        const bool parallel = xyz != nullptr && depth < kParallelDepth && !rest_a.empty() && !b.empty() &&
                              std::min(rest_a.size(), b.size()) >= kParallelVertices;
        if (parallel) {
            std::vector<Node> tree_a, tree_b;
            std::vector<int> order_a, order_b;
            std::thread worker([&]() { dissect(std::move(rest_a), tree_a, order_a, depth + 1); });
            dissect(std::move(b), tree_b, order_b, depth + 1);
            worker.join();
            for (auto* piece : {&tree_a, &tree_b}) {
                const auto& order_piece = piece == &tree_a ? order_a : order_b;
                const int node_shift = (int)tree_out.size(), start_shift = (int)order_out.size();
                for (Node nd : *piece) {
                    nd.start += start_shift;
                    for (int& c : nd.children) c += node_shift;
                    if (nd.parent >= 0) nd.parent += node_shift;
                    tree_out.push_back(std::move(nd));
                }
                order_out.insert(order_out.end(), order_piece.begin(), order_piece.end());
                children.push_back((int)tree_out.size() - 1);
            }
        } else {
            if (!rest_a.empty()) children.push_back(dissect(std::move(rest_a), tree_out, order_out, depth + 1));
            if (!b.empty()) children.push_back(dissect(std::move(b), tree_out, order_out, depth + 1));
        }
        std::sort(sep.begin(), sep.end());
        Node node;
        node.start = (int)order_out.size();
        node.count = (int)sep.size();
        node.children = children;
        order_out.insert(order_out.end(), sep.begin(), sep.end());
        tree_out.push_back(node);
        const int id = (int)tree_out.size() - 1;
        for (int c : children) tree_out[c].parent = id;
        return id;
    }

    int dissect(std::vector<int> verts) { return dissect(std::move(verts), tree, order, 0); }
};

// Symbolic analysis of a dissection: each node's off-diagonal rows are its columns' later
// neighbours plus its children's off-diagonal rows past its own columns; its level is its height
// above the leaves. The nodes of one level depend only on the levels below, so each level's
// nodes run across host threads (each node's rows sorted and deduplicated on its own).
void symbolic(Analysis& A, const std::vector<int>& adj_off, const std::vector<int>& adj) {
    const int ns = (int)A.nodes.size();
    // Heights (the nodes are in postorder: children first), then the nodes bucketed by height.
    std::vector<int> height(ns, 0);
    int top = 0;
    for (int s = 0; s < ns; ++s) {
        int level = 0;
        for (int c : A.nodes[s].children) level = std::max(level, height[c] + 1);
        height[s] = level;
        top = std::max(top, level);
    }
    std::vector<int> first(top + 2, 0), bucket(ns);
    for (int s = 0; s < ns; ++s) ++first[height[s] + 1];
    for (int l = 0; l <= top; ++l) first[l + 1] += first[l];
    {
        std::vector<int> fill(first.begin(), first.end() - 1);
        for (int s = 0; s < ns; ++s) bucket[fill[height[s]]++] = s;
    }
    for (int l = 0; l <= top; ++l) {
        const int* nodes = bucket.data() + first[l];
        const long long count = first[l + 1] - first[l];
        parallel_range(count, A.n > (1 << 16), [&](long long lo, long long hi) {
            std::vector<int> rows;
            for (long long i = lo; i < hi; ++i) {
                Node& node = A.nodes[nodes[i]];
                const int end = node.start + node.count;
                rows.clear();
                for (int j = node.start; j < end; ++j) {
                    const int old = A.perm[j];
                    for (int e = adj_off[old]; e < adj_off[old + 1]; ++e) {
                        const int r = A.iperm[adj[e]];
                        if (r >= end) rows.push_back(r);
                    }
                }
                for (int c : node.children)
                    for (int r : A.nodes[c].off_rows)
                        if (r >= end) rows.push_back(r);
                std::sort(rows.begin(), rows.end());
                rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
                node.off_rows.assign(rows.begin(), rows.end());
                node.level = l;
            }
        });
    }
    A.levels = top + 1;
    A.factor_entries = 0;
    for (const Node& node : A.nodes)
        A.factor_entries += (long long)node.count * node.count + (long long)node.off_rows.size() * node.count;
}

// Level amalgamation. Each tree level costs the solves one dependent launch per direction (a
// few microseconds of launch and pipeline latency however little work the level holds), so whole
// levels above the leaves are merged into their parents while that is cheap: merging the nodes
// of level l into their parents at l + 1 makes each parent one dense supernode of its own and
// the merged children's columns (its off-diagonal rows stay the parent's), adding explicit zeros
// to the stored factor. The cheapest level goes first, as long as it adds at most kMergeValues
// stored values (about 12 us of float64 tensor work for a 64-column pass, against the ~20 us the
// two launches cost) and the factor stays within kMergeGrowth of its unmerged size. Columns of a
// merged node are renumbered to be contiguous (the merged children's columns, then the parent's):
// siblings' separators never share an edge, so this changes no fill outside the merged fronts.
constexpr long long kMergeValues = 1750000;
constexpr double kMergeGrowth = 1.3;

void amalgamate(Analysis& A, const std::vector<int>& adj_off, const std::vector<int>& adj) {
    const int ns = (int)A.nodes.size();
    if (A.levels < 3) return;
    auto padded = [](long long c) { return (c + 7) / 8 * 8; };
    std::vector<long long> nc(ns), noff(ns);
    std::vector<std::vector<int>> kids(ns), cols_of(ns);
    std::vector<char> alive(ns, 1);
    long long total = 0;
    for (int s = 0; s < ns; ++s) {
        nc[s] = A.nodes[s].count;
        noff[s] = (long long)A.nodes[s].off_rows.size();
        kids[s] = A.nodes[s].children;
        cols_of[s].assign(1, s);
        total += (nc[s] + noff[s]) * padded(nc[s]);
    }
    const long long limit = (long long)(kMergeGrowth * (double)total);
    std::vector<int> level(ns, 0);
    bool merged_any = false;
    for (;;) {
        int top = 0;
        for (int s = 0; s < ns; ++s) {
            if (!alive[s]) continue;
            int l = 0;
            for (int c : kids[s]) l = std::max(l, level[c] + 1);
            level[s] = l;
            top = std::max(top, l);
        }
        // The merge cost of every level 1 .. top - 1 (leaves stay: merging them is dense work).
        std::vector<long long> delta(top + 1, 0);
        std::vector<char> candidate(top + 1, 0);
        for (int p = 0; p < ns; ++p) {
            if (!alive[p] || level[p] < 2) continue;
            const int l = level[p] - 1;
            long long m = nc[p], before = (nc[p] + noff[p]) * padded(nc[p]);
            bool any = false;
            for (int c : kids[p])
                if (level[c] == l) {
                    m += nc[c];
                    before += (nc[c] + noff[c]) * padded(nc[c]);
                    any = true;
                }
            if (!any) continue;
            candidate[l] = 1;
            delta[l] += (m + noff[p]) * padded(m) - before;
        }
        int best = -1;
        for (int l = 1; l < top; ++l)
            if (candidate[l] && (best < 0 || delta[l] < delta[best])) best = l;
        if (best < 0 || delta[best] > kMergeValues || total + delta[best] > limit) break;
        for (int p = 0; p < ns; ++p) {
            if (!alive[p] || level[p] != best + 1) continue;
            std::vector<int> next, absorbed;
            for (int c : kids[p]) {
                if (level[c] == best) {
                    nc[p] += nc[c];
                    alive[c] = 0;
                    absorbed.insert(absorbed.end(), cols_of[c].begin(), cols_of[c].end());
                    next.insert(next.end(), kids[c].begin(), kids[c].end());
                } else {
                    next.push_back(c);
                }
            }
            absorbed.insert(absorbed.end(), cols_of[p].begin(), cols_of[p].end());
            cols_of[p] = std::move(absorbed);
            kids[p] = std::move(next);
        }
        total += delta[best];
        merged_any = true;
    }
    if (!merged_any) return;
    // Renumber: the surviving nodes in postorder (children first, each subtree contiguous), each
    // node's columns those of the original nodes merged into it.
    std::vector<int> order;
    order.reserve(A.n);
    std::vector<Node> tree;
    std::function<int(int)> emit = [&](int s) -> int {
        std::vector<int> children;
        for (int c : kids[s]) children.push_back(emit(c));
        Node node;
        node.start = (int)order.size();
        for (int o : cols_of[s])
            for (int j = 0; j < A.nodes[o].count; ++j) order.push_back(A.perm[A.nodes[o].start + j]);
        node.count = (int)order.size() - node.start;
        node.children = children;
        tree.push_back(node);
        const int id = (int)tree.size() - 1;
        for (int c : children) tree[c].parent = id;
        return id;
    };
    for (int s = 0; s < ns; ++s)
        if (alive[s] && A.nodes[s].parent < 0) emit(s);
    A.perm = std::move(order);
    A.nodes = std::move(tree);
    for (int i = 0; i < A.n; ++i) A.iperm[A.perm[i]] = i;
    symbolic(A, adj_off, adj);
}

// `block` > 1: the operator's rows come in groups of `block` consecutive rows, one group a mesh
// vertex (xyz holds n / block points), as in a system of tangent vectors. The dissection then runs
// over the vertices' graph and every vertex's rows stay together, consecutive in the ordering.
int analyse(int n, std::vector<int> offsets, std::vector<int> columns, const float* xyz,
            int leaf_size, Analysis* out, int block = 1) {
    Analysis& A = *out;
    A.n = n;
    A.offsets = std::move(offsets);
    A.columns = std::move(columns);
    // Adjacency without the diagonal, for the separators and the components: each row's count,
    // their prefix sum, then each row's entries in place (rows across host threads).
    std::vector<int> adj_off(n + 1, 0);
    const bool large = A.columns.size() > (1u << 18);
    parallel_range(n, large, [&](long long lo, long long hi) {
        for (long long i = lo; i < hi; ++i) {
            int count = 0;
            for (int e = A.offsets[i]; e < A.offsets[i + 1]; ++e) count += A.columns[e] != (int)i;
            adj_off[i + 1] = count;
        }
    });
    for (int i = 0; i < n; ++i) adj_off[i + 1] += adj_off[i];
    std::vector<int> adj(adj_off[n]);
    parallel_range(n, large, [&](long long lo, long long hi) {
        for (long long i = lo; i < hi; ++i) {
            int at = adj_off[i];
            for (int e = A.offsets[i]; e < A.offsets[i + 1]; ++e)
                if (A.columns[e] != (int)i) adj[at++] = A.columns[e];
        }
    });
    if (leaf_size <= 0) leaf_size = kDefaultLeafSize;
    if (block > 1) {
        const int nv = n / block;
        std::vector<int> vadj_off(nv + 1, 0), vadj, seen(nv, -1);
        for (int v = 0; v < nv; ++v) {
            for (int r = block * v; r < block * v + block; ++r)
                for (int e = A.offsets[r]; e < A.offsets[r + 1]; ++e) {
                    const int u = A.columns[e] / block;
                    if (u != v && seen[u] != v) {
                        seen[u] = v;
                        vadj.push_back(u);
                    }
                }
            vadj_off[v + 1] = (int)vadj.size();
        }
        Dissector D(vadj_off, vadj, xyz, nv, std::max(1, leaf_size / block));
        std::vector<int> all(nv);
        std::iota(all.begin(), all.end(), 0);
        D.dissect(std::move(all));
        A.perm.resize(n);
        for (int p = 0; p < nv; ++p)
            for (int b = 0; b < block; ++b) A.perm[block * p + b] = block * D.order[p] + b;
        A.nodes = std::move(D.tree);
        for (Node& node : A.nodes) {
            node.start *= block;
            node.count *= block;
        }
    } else {
        Dissector D(adj_off, adj, xyz, n, leaf_size);
        std::vector<int> all(n);
        std::iota(all.begin(), all.end(), 0);
        D.dissect(std::move(all));
        A.perm = std::move(D.order);
        A.nodes = std::move(D.tree);
    }
    A.iperm.assign(n, 0);
    for (int i = 0; i < n; ++i) A.iperm[A.perm[i]] = i;
    symbolic(A, adj_off, adj);
    amalgamate(A, adj_off, adj);
    // Components (for pinning a singular operator): each vertex's component label and the last
    // vertex of each in the new order.
    A.component_last.assign(n, 0);
    std::vector<int> comp(n, -1);
    std::vector<int> queue;
    A.n_components = 0;
    for (int seed = 0; seed < n; ++seed) {
        if (comp[seed] >= 0) continue;
        comp[seed] = A.n_components++;
        queue.assign(1, seed);
        int last = seed;
        for (size_t h = 0; h < queue.size(); ++h) {
            const int v = queue[h];
            if (A.iperm[v] > A.iperm[last]) last = v;
            for (int e = adj_off[v]; e < adj_off[v + 1]; ++e)
                if (comp[adj[e]] < 0) {
                    comp[adj[e]] = comp[seed];
                    queue.push_back(adj[e]);
                }
        }
        A.component_last[last] = 1;
    }
    A.component = std::move(comp);
    return OB_OK;
}

// ------------------------------------------------------------------------------------------
// Numeric factorisation (host, multifrontal over the dissection tree).
// ------------------------------------------------------------------------------------------

struct HostFactor {
    std::vector<std::vector<double>> inv;     // per node: nc x nc row-major inverse of L11
    std::vector<std::vector<double>> off;     // per node: (m - nc) x nc row-major -L21 L11^-1
    std::vector<std::vector<double>> update;  // per node: (m - nc)^2 column-major, for the parent
    std::vector<char> pinned;                 // per new index: identity row (pinned / empty)
};

// Fronts from this size up (the ones at the top of the tree, factored after the parallel
// subtrees) spread their dense work over host threads (parallel_range).
constexpr int kThreadedFront = 384;

// Dense partial Cholesky of the m x m column-major front F (lower part used): the first nc
// columns are factored in place (L11, L21) and F22 becomes the Schur complement.
// C -= A B^T on column-major blocks: C(i, j) at C[j * ldc + i] for i < M, j < N, A(i, kk) at
// A[kk * lda + i], B(j, kk) at B[kk * ldb + j], kk < K. Register-blocked 8 x 4: each inner step
// loads 8 consecutive rows of A's column kk and 4 entries of B's column kk and does 32
// multiply-adds in registers (eight 4-wide vector accumulators), so the dense host work of the
// factorisation streams from cache instead of re-reading a column per axpy. The sum over kk runs
// in order for every entry.
typedef double v4d __attribute__((vector_size(32)));

inline void gemm_block_8x4(double* C, int ldc, const double* A, int lda, const double* B, int ldb, int K) {
    v4d acc[4][2] = {};
    for (int kk = 0; kk < K; ++kk) {
        v4d a0, a1;
        __builtin_memcpy(&a0, A + (size_t)kk * lda, sizeof(v4d));
        __builtin_memcpy(&a1, A + (size_t)kk * lda + 4, sizeof(v4d));
        const double* b = B + (size_t)kk * ldb;
#pragma GCC unroll 4
        for (int c = 0; c < 4; ++c) {
            const v4d bc = {b[c], b[c], b[c], b[c]};
            acc[c][0] += a0 * bc;
            acc[c][1] += a1 * bc;
        }
    }
#pragma GCC unroll 4
    for (int c = 0; c < 4; ++c) {
        double* out = C + (size_t)c * ldc;
        v4d o0, o1;
        __builtin_memcpy(&o0, out, sizeof(v4d));
        __builtin_memcpy(&o1, out + 4, sizeof(v4d));
        o0 -= acc[c][0];
        o1 -= acc[c][1];
        __builtin_memcpy(out, &o0, sizeof(v4d));
        __builtin_memcpy(out + 4, &o1, sizeof(v4d));
    }
}

void gemm_nt_minus(double* C, int ldc, const double* A, int lda, const double* B, int ldb, int M, int N,
                   int K) {
    constexpr int kR = 8, kC = 4;
    for (int j0 = 0; j0 < N; j0 += kC) {
        const int nj = std::min(kC, N - j0);
        for (int i0 = 0; i0 < M; i0 += kR) {
            const int ni = std::min(kR, M - i0);
            if (ni == kR && nj == kC) {
                gemm_block_8x4(C + (size_t)j0 * ldc + i0, ldc, A + i0, lda, B + j0, ldb, K);
                continue;
            }
            double acc[kC][kR] = {};
            for (int kk = 0; kk < K; ++kk) {
                const double* a = A + (size_t)kk * lda + i0;
                const double* b = B + (size_t)kk * ldb + j0;
                for (int c = 0; c < nj; ++c)
                    for (int r = 0; r < ni; ++r) acc[c][r] += a[r] * b[c];
            }
            for (int c = 0; c < nj; ++c) {
                double* out = C + (size_t)(j0 + c) * ldc + i0;
                for (int r = 0; r < ni; ++r) out[r] -= acc[c][r];
            }
        }
    }
}

bool partial_cholesky(double* F, int m, int nc) {
    constexpr int kBlock = 48;
    for (int j0 = 0; j0 < nc; j0 += kBlock) {
        const int j1 = std::min(nc, j0 + kBlock);
        // Factor the panel columns [j0, j1) (already updated by earlier panels).
        for (int j = j0; j < j1; ++j) {
            double* cj = F + (size_t)j * m;
            const double d = cj[j];
            if (!(d > 0.0)) return false;
            const double r = std::sqrt(d);
            cj[j] = r;
            const double inv = 1.0 / r;
            for (int i = j + 1; i < m; ++i) cj[i] *= inv;
            for (int k = j + 1; k < j1; ++k) {
                double* ck = F + (size_t)k * m;
                const double f = cj[k];
                if (f != 0.0)
                    for (int i = k; i < m; ++i) ck[i] -= cj[i] * f;
            }
        }
        // Update every later column with the panel: F[k:, k] -= L[k:, j0:j1] L[k, j0:j1]^T, in
        // blocks of 4 columns (rows from the block's first column down; the few entries above
        // the diagonal it also writes are never read). On a large front the blocks are split
        // over host threads in ranges of equal work (a column's work falls with its index).
        const int blocks = (m - j1 + 3) / 4;
        auto update = [&](int b0, int b1) {
            for (int b = b0; b < b1; ++b) {
                const int k0 = j1 + 4 * b, nk = std::min(4, m - k0);
                gemm_nt_minus(F + (size_t)k0 * m + k0, m, F + (size_t)j0 * m + k0, m, F + (size_t)j0 * m + k0, m,
                              m - k0, nk, j1 - j0);
            }
        };
        const int parts = m >= kThreadedFront ? std::min(host_threads(), std::max(1, blocks / 8)) : 1;
        if (parts <= 1) {
            update(0, blocks);
        } else {
            // Block b costs about (m - j1 - 4 b); cut where the running cost crosses p / parts.
            std::vector<int> cut(parts + 1, blocks);
            cut[0] = 0;
            const double total = 0.5 * (double)blocks * (2.0 * (m - j1) - 4.0 * (blocks - 1));
            double run = 0.0;
            int next = 1;
            for (int b = 0; b < blocks && next < parts; ++b) {
                run += (double)(m - j1 - 4 * b);
                if (run >= total * next / parts) cut[next++] = b + 1;
            }
            run_parts(parts, [&](int p) { update(cut[p], cut[p + 1]); });
        }
    }
    return true;
}

int factor_node(const Analysis& A, const double* values, int s, bool singular, HostFactor& H,
                std::vector<int>& local) {
    const Node& node = A.nodes[s];
    const int nc = node.count, noff = (int)node.off_rows.size(), m = nc + noff;
    const int end = node.start + nc;
    std::vector<double> F((size_t)m * m, 0.0);
    for (int j = 0; j < nc; ++j) local[node.start + j] = j;
    for (int r = 0; r < noff; ++r) local[node.off_rows[r]] = nc + r;
    // Assemble the operator's entries of the own columns (lower part, rows in R_s).
    for (int j = node.start; j < end; ++j) {
        const int old = A.perm[j];
        const bool pin = H.pinned[j];
        const int lj = j - node.start;
        if (pin) {
            F[(size_t)lj * m + lj] = 1.0;
            continue;
        }
        for (int e = A.offsets[old]; e < A.offsets[old + 1]; ++e) {
            const int r = A.iperm[A.columns[e]];
            if (r < j || H.pinned[r]) continue;
            F[(size_t)lj * m + local[r]] += values[e];
        }
    }
    // Extend-add the children's update matrices.
    for (int c : node.children) {
        const Node& ch = A.nodes[c];
        const int cm = (int)ch.off_rows.size();
        const std::vector<double>& U = H.update[c];
        for (int b = 0; b < cm; ++b) {
            const int lb = local[ch.off_rows[b]];
            for (int a = b; a < cm; ++a) {
                const int la = local[ch.off_rows[a]];
                const int row = std::max(la, lb), colm = std::min(la, lb);
                F[(size_t)colm * m + row] += U[(size_t)b * cm + a];
            }
        }
        H.update[c].clear();
        H.update[c].shrink_to_fit();
    }
    if (!partial_cholesky(F.data(), m, nc)) return OB_ERR_INDEFINITE;
    // Inverse of L11 (lower triangular), row-major, by block forward substitution over rows:
    // rows [i0, i1) of X = L^-1 are first reduced by the rows above them (X[I, :] -= L[I, 0:i0]
    // X[0:i0, :], one blocked product, threaded over columns on a large front), then solved
    // row by row against the diagonal block.
    constexpr int kInvBlock = 48;
    std::vector<double> inv((size_t)nc * nc, 0.0);
    for (int i = 0; i < nc; ++i) inv[(size_t)i * nc + i] = 1.0;
    for (int i0 = 0; i0 < nc; i0 += kInvBlock) {
        const int i1 = std::min(nc, i0 + kInvBlock);
        if (i0 > 0) {
            // Transposed view: C(c, i) = inv[i][c] -= sum_kk inv[kk][c] L[i][kk] for the columns
            // c < i0 that rows above can reach; threaded over columns on a large front.
            parallel_range(i0, m >= kThreadedFront, [&](long long begin, long long end) {
                gemm_nt_minus(inv.data() + (size_t)i0 * nc + begin, nc, inv.data() + begin, nc, F.data() + i0, m,
                              (int)(end - begin), i1 - i0, i0);
            });
        }
        for (int i = i0; i < i1; ++i) {
            double* xi = inv.data() + (size_t)i * nc;
            for (int kk = i0; kk < i; ++kk) {
                const double l = F[(size_t)kk * m + i];
                if (l == 0.0) continue;
                const double* xk = inv.data() + (size_t)kk * nc;
                for (int c = 0; c <= kk; ++c) xi[c] -= l * xk[c];
            }
            const double d = F[(size_t)i * m + i];
            for (int c = 0; c <= i; ++c) xi[c] /= d;
        }
    }
    // The off-diagonal block the solves use, G = -L21 L11^-1 (row r: minus the row of L21 times
    // the lower-triangular inverse): with it both of a node's products in each direction read
    // only inputs that are final when its level starts -- forward y1 = L11^-1 b1 and b2 += G b1,
    // backward x1 = L11^-T y1 + G^T x2 -- so a tree level is one launch a direction.
    // Transposed view: C(i, r) = G[r][i] -= sum_k inv[k][i] L21[r][k] (L21[r][k] = F column k,
    // row nc + r), for 8 entries i at a time over k >= i only (inv is lower triangular); threaded
    // over rows of G on a large front.
    std::vector<double> G((size_t)noff * nc, 0.0);
    parallel_range(noff, m >= kThreadedFront, [&](long long begin, long long end) {
        for (int i0 = 0; i0 < nc; i0 += 8)
            gemm_nt_minus(G.data() + (size_t)begin * nc + i0, nc, inv.data() + (size_t)i0 * nc + i0, nc,
                          F.data() + (size_t)i0 * m + nc + begin, m, std::min(8, nc - i0), (int)(end - begin),
                          nc - i0);
    });
    H.inv[s] = std::move(inv);
    H.off[s] = std::move(G);
    std::vector<double> U((size_t)noff * noff);
    for (int b = 0; b < noff; ++b)
        for (int a = b; a < noff; ++a) U[(size_t)b * noff + a] = F[(size_t)(nc + b) * m + nc + a];
    H.update[s] = std::move(U);
    (void)singular;
    return OB_OK;
}

int numeric(const Analysis& A, const double* values, bool singular, HostFactor* out) {
    HostFactor& H = *out;
    const int ns = (int)A.nodes.size();
    H.inv.assign(ns, {});
    H.off.assign(ns, {});
    H.update.assign(ns, {});
    H.pinned.assign(A.n, 0);
    for (int i = 0; i < A.n; ++i) {
        const int old = A.perm[i];
        bool empty = true;
        for (int e = A.offsets[old]; e < A.offsets[old + 1]; ++e)
            if (A.columns[e] == old && values[e] != 0.0) empty = false;
        if (empty || (singular && A.component_last[old])) H.pinned[i] = 1;
    }
    // Subtrees below a cut level are factored in parallel, the rest in postorder.
    const unsigned threads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    int cut = A.levels - 1;
    while (cut > 0) {
        int count = 0;
        for (const Node& nd : A.nodes)
            if (nd.level == cut - 1 && (nd.parent < 0 || A.nodes[nd.parent].level >= cut)) ++count;
        if (count >= (int)threads * 2) break;
        --cut;
    }
    // Roots of the parallel subtrees: nodes below `cut` whose parent is at or above it.
    std::vector<int> roots;
    for (int s = 0; s < ns; ++s)
        if (A.nodes[s].level < cut && (A.nodes[s].parent < 0 || A.nodes[A.nodes[s].parent].level >= cut))
            roots.push_back(s);
    std::vector<int> status(roots.size(), OB_OK);
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        std::vector<int> local(A.n, -1);
        for (;;) {
            const size_t i = next.fetch_add(1);
            if (i >= roots.size()) break;
            // Postorder of the subtree rooted at roots[i]: its nodes are a contiguous index range
            // ending at the root (the tree was appended in postorder).
            const int root = roots[i];
            int first = root;
            std::function<void(int)> lowest = [&](int v) {
                first = std::min(first, v);
                for (int c : A.nodes[v].children) lowest(c);
            };
            lowest(root);
            for (int s = first; s <= root && status[i] == OB_OK; ++s)
                status[i] = factor_node(A, values, s, singular, H, local);
        }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
    for (int st : status)
        if (st) return st;
    std::vector<int> local(A.n, -1);
    for (int s = 0; s < ns; ++s) {
        if (A.nodes[s].level < cut) continue;
        int st = factor_node(A, values, s, singular, H, local);
        if (st) return st;
    }
    return OB_OK;
}

// ------------------------------------------------------------------------------------------
// Device factor and the level-scheduled solve.
// ------------------------------------------------------------------------------------------

// One output tile of a batched dense product: out rows [r0, r0 + rows) of a block whose matrix
// is M (row-major, leading dimension ld, or its transpose when trans), times input rows
// [k0, k1) of the inner dimension (a long inner dimension is split over several tiles).
enum TileOp : int { kAssign = 0, kAtomicSub = 1, kSub = 2, kAtomicAdd = 3 };

struct Tile {
    long long m;     // offset of the matrix in the value buffer
    int ld, trans;   // leading dimension; 1 when the matrix is read transposed
    int r0, rows;    // output rows [r0, r0 + rows) of the block
    int k0, k1;      // inner-dimension range of this tile
    int in_base;     // input row index: in_rows == -1 -> in_base + kk, else idx[in_rows + kk]
    int in_rows;
    int out_base;    // output row index: out_rows == -1 -> out_base + i, else idx[out_rows + i]
    int out_rows;
    int op;          // TileOp
    // Known-zero structure of the block, used to skip whole inner steps: 0 dense; 1 lower
    // triangular (entry (i, kk) zero for kk > i: the forward L11^-1); 2 the backward
    // [L11^-1; G]^T (entry (i, kk) zero for kk < i while kk < tri_k = nc).
    int tri, tri_k;
    int node;  // the supernode the tile belongs to (a forward pass may skip inactive nodes)
};

constexpr int kTileRows = 64;   // output rows per tile
constexpr int kWorkSets = 6;    // independent work-buffer sets a factor holds
constexpr int kTileCols = 64;   // right-hand-side columns per tile (the wide form)
constexpr int kTileColsNarrow = 32;  // the narrow form: twice the CTAs, half the columns each
// Batches of 9-16 columns: 16-column tiles (a 32-column tile computed 16 padding columns; the
// packed batch of 256 meshes at 16 columns: 226 k -> 319 k solves/s).
constexpr int kTileColsSixteen = 16;
// Inner-dimension step staged in shared memory. 16 (two stages, 39 KB, 4 CTAs per SM) measured
// 0.82 ms a pass on the 131k torus at 64 columns, against 1.11 ms for 32 (74 KB, 3 CTAs per SM).
constexpr int kTileK = 16;
constexpr int kSplitK = 64;  // a split tile's inner-dimension range (32 measured slower: more atomics)
constexpr int kTileThreads = 128;  // the narrow form's CTA: four warps, each a 16-row strip
// The wide form's CTA: eight warps, a 16-row strip of 32 of the 64 columns each, so the matrix
// block staged once feeds 64 columns while a warp holds half the accumulators (64 registers).
constexpr int kTileThreadsWide = 256;
template <int TC>
constexpr int tile_threads() { return TC == kTileCols ? kTileThreadsWide : kTileThreads; }
// Resident CTAs of the 64-column product an SM: three of eight warps at up to 80 registers a
// thread, two stages of 19.5 KB each (the 131k torus at 64 columns, a pass: 0.397 ms; four CTAs
// at 64 registers 0.401 ms; the four-warp CTA, five an SM at 96 registers, 0.428 ms; three
// stages at three CTAs 0.410 ms).
constexpr int kTileCtasPerSm = 3;
// Resident CTAs of the 32-column product an SM: four warps at up to 73 registers a thread, two
// stages of 15 KB (seven fill the shared memory). The tuner picks this form for every level of the
// 131k torus at 64 columns: 0.381 ms a pass, against 0.392 ms at six an SM and 0.398 ms at eight
// (64 registers, with spills).
constexpr int kTileCtasPerSmNarrow = 7;
// Shared rows of 72 doubles (a transposed matrix block's 64 output rows, a 64-column input row):
// the 8 x 4 fragment loads of a warp then touch every 8-byte bank pair exactly twice (the minimum
// for 256 bytes); 40 for a 32-column input row.
constexpr int kLd = kTileRows + 8;
template <int TC>
constexpr int input_ld() { return TC + 8; }

// 16-byte asynchronous global -> shared copies; bytes < 16 zero-fills the rest (0: all zeros, and
// the source is not read). Both read through L2 only: a factor block is read once per tile, and
// with the shared-memory carveout at its maximum the L1 left over is small (caching the factor
// there, `.ca`, measured 0.478 against 0.444 ms a pass); the work vectors are also updated by
// other launches' atomics.
__device__ __forceinline__ void copy16(void* smem, const void* gmem, int bytes) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void copy16_l2(void* smem, const void* gmem, int bytes) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void copy_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void copy_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Shared staging of one inner-dimension step: the matrix block (row-major [64][kLdK] for a
// row-major matrix, k-major [16][kLd] for a transposed one) and the 16 gathered input rows.
constexpr int kLdK = kTileK + 4;  // row-major staging: fragment loads touch each bank pair twice
template <int TC>
struct Stage {
    double a[kTileRows * kLdK > kTileK * kLd ? kTileRows * kLdK : kTileK * kLd];
    double b[kTileK * input_ld<TC>()];
};

// One 64 x TC output tile for a CTA of four 16-row strips of warps, each strip one warp (TC = 32,
// 2 x 4 float64 MMA tiles) or two (TC = 64: a warp each 32 of the columns, 2 x 4 MMA tiles);
// strips rather than quadrants, so a strip of padding rows, or of the zero triangle of L11^-1
// over an inner step, is skipped whole. The tile's matrix block and its
// gathered input rows are copied 16 inner steps at a time into shared memory with asynchronous
// 16-byte copies (zero-filled at the edges), two stages: the next step's copies, issued after the
// step's one barrier, overlap the current step's MMAs. The output is assigned, subtracted, or
// added atomically per the tile's op. `k` (the column stride) is even and every block row starts
// on 16 bytes, so every copy is aligned. `in` and `out` are the same stacked work buffer: the rows
// a launch's tiles read are never rows any tile of that launch writes.
template <int TC>
struct TileOps {
    static constexpr int kThreads = tile_threads<TC>();
    static constexpr int kGroups = kThreads / kTileThreads;  // column groups of warps
    static constexpr int kJ = TC / 8 / kGroups;               // 8-column MMA tiles a warp holds
    static constexpr int kLdB = input_ld<TC>();
    // The matrix block is 64 x kTileK doubles in 16-byte chunks, kChunks per thread; the input
    // block kTileK x TC, kChunksB per thread.
    static constexpr int kChunks = kTileRows * kTileK / 2 / kThreads;
    static constexpr int kChunksB = TC * kTileK / 2 / kThreads;
    using Acc = double[2][kJ][2];

    __device__ static int steps(const Tile& t) { return (t.k1 - t.k0 + kTileK - 1) / kTileK; }

    // The input rows of this thread's chunks of the inner step from kb (-1 past the inner range).
    __device__ static void input_rows(const Tile& t, int kb, const int* __restrict__ idx, int* r) {
#pragma unroll
        for (int q = 0; q < kChunksB; ++q) {
            const int kk = (threadIdx.x + q * kThreads) / (TC / 2);
            r[q] = kb + kk < t.k1 ? (t.in_rows < 0 ? t.in_base + kb + kk : idx[t.in_rows + kb + kk]) : -1;
        }
    }

    // Issues (and commits as one group) the copies of the inner step from kb into a stage.
    __device__ static void issue(const Tile& t, int c0, int kb, const int* in_row, const double* __restrict__ vals,
                                 const double* in, int k, Stage<TC>& s) {
        const double* M = vals + t.m;
#pragma unroll
        for (int q = 0; q < kChunks; ++q) {
            const int chunk = threadIdx.x + q * kThreads;
            if (t.trans) {
                // Row kk of the stored matrix, elements r0 + 2 c .. + 1: k-major staging.
                const int kk = chunk / (kTileRows / 2), c2 = 2 * (chunk % (kTileRows / 2));
                const int valid = (kb + kk < t.k1) ? max(0, min(2, t.rows - c2)) : 0;
                const double* src = valid ? M + (size_t)(kb + kk) * t.ld + t.r0 + c2 : M;
                copy16(&s.a[kk * kLd + c2], src, 8 * valid);
            } else {
                // Row i of the block, elements kb + 2 c .. + 1: row-major staging.
                const int i = chunk / (kTileK / 2), c2 = 2 * (chunk % (kTileK / 2));
                const int valid = (i < t.rows) ? max(0, min(2, t.k1 - kb - c2)) : 0;
                const double* src = valid ? M + (size_t)(t.r0 + i) * t.ld + kb + c2 : M;
                copy16(&s.a[i * kLdK + c2], src, 8 * valid);
            }
        }
#pragma unroll
        for (int q = 0; q < kChunksB; ++q) {
            const int chunk = threadIdx.x + q * kThreads;
            // Input rows: row kk of the step, columns c0 + 2 c .. + 1.
            const int kk = chunk / (TC / 2), c2 = 2 * (chunk % (TC / 2));
            int valid = 0;
            const double* src = in;
            if (in_row[q] >= 0 && c0 + c2 < k) {
                src = in + (size_t)in_row[q] * k + c0 + c2;
                valid = 16;
            }
            copy16_l2(&s.b[kk * kLdB + c2], src, valid);
        }
        copy_commit();
    }

    // The output rows of this thread's accumulator rows (-1 past the tile).
    __device__ static int strip() { return ((threadIdx.x >> 5) & 3) * 16; }
    __device__ static int group_column() { return (threadIdx.x >> 7) * (TC / kGroups); }

    __device__ static void output_rows(const Tile& t, const int* __restrict__ idx, int* out_row) {
        const int lane = threadIdx.x & 31, wr = strip();
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int local = wr + 8 * i + (lane >> 2);
            out_row[i] = local >= t.rows ? -1
                         : (t.out_rows < 0 ? t.out_base + t.r0 + local : idx[t.out_rows + t.r0 + local]);
        }
    }

    // The MMAs of the inner step from kb out of its stage. A strip skips a whole inner step when
    // all its products are known zeros: padding rows past the tile, or the zero triangle of
    // L11^-1 (the decision is warp-uniform and taken outside the unrolled step, which stays
    // branch-free).
    __device__ static void compute(const Tile& t, int kb, const Stage<TC>& s, Acc& acc) {
        const int lane = threadIdx.x & 31, wr = strip(), cg = group_column();
        const int fr = lane >> 2, fk = lane & 3;  // fragment coordinates
        const int row_lo = t.r0 + wr, row_hi = row_lo + 15;
        const bool zero = wr >= t.rows || (t.tri == 1 && kb > row_hi) ||
                          (t.tri == 2 && kb + kTileK - 1 < row_lo && kb + kTileK - 1 < t.tri_k);
        if (zero) return;
#pragma unroll
        for (int k4 = 0; k4 < kTileK; k4 += 4) {
            double a[2], b[kJ];
            if (t.trans) {
#pragma unroll
                for (int i = 0; i < 2; ++i) a[i] = s.a[(k4 + fk) * kLd + wr + 8 * i + fr];
            } else {
#pragma unroll
                for (int i = 0; i < 2; ++i) a[i] = s.a[(wr + 8 * i + fr) * kLdK + k4 + fk];
            }
#pragma unroll
            for (int j = 0; j < kJ; ++j) b[j] = s.b[(k4 + fk) * kLdB + cg + 8 * j + fr];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < kJ; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
    }

    __device__ static void clear(Acc& acc) {
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < kJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    }

    // Applies the tile's op to its outputs.
    __device__ static void store(const Tile& t, int c0, const int* out_row, double* out, int k, const Acc& acc) {
        const int fk = threadIdx.x & 3, cg = group_column();
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = out_row[i];
            if (r < 0) continue;
#pragma unroll
            for (int j = 0; j < kJ; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int c = c0 + cg + 8 * j + 2 * fk + h;
                    if (c >= k) continue;
                    double* o = out + (size_t)r * k + c;
                    const double v = acc[i][j][h];
                    switch (t.op) {
                        case kAssign: *o = v; break;
                        case kAtomicSub: atomicAdd(o, -v); break;
                        case kSub: *o = __ldcg(o) - v; break;
                        default: atomicAdd(o, v); break;
                    }
                }
        }
    }
};

template <int TC>
__device__ __forceinline__ void tile_product(const Tile& t, int k0, int c0, const double* __restrict__ vals,
                                             const int* __restrict__ idx,
                                             const double* in, double* out, int k, Stage<TC>* stage) {
    using Ops = TileOps<TC>;
    typename Ops::Acc acc;
    Ops::clear(acc);
    // Inner steps from k0 (the tile's own, or past a zero Y block: first_inner).
    const int steps = (t.k1 - k0 + kTileK - 1) / kTileK;
    if (steps <= 0) {
        // Nothing to multiply: an assigned output is zero, an accumulated one unchanged.
        if (t.op == kAssign) {
            int rows_out[2];
            Ops::output_rows(t, idx, rows_out);
            Ops::store(t, c0, rows_out, out, k, acc);
        }
        return;
    }
    // The input rows of a step's chunks are read one step ahead of the copies that use them, so
    // a gathered index's load latency is not paid in front of every step's copies.
    int first_rows[Ops::kChunksB], next_rows[Ops::kChunksB];
    Ops::input_rows(t, k0, idx, first_rows);
    Ops::issue(t, c0, k0, first_rows, vals, in, k, stage[0]);
    if (steps > 1) Ops::input_rows(t, k0 + kTileK, idx, next_rows);
    // The output rows, read before the products so the epilogue does not wait on them.
    int out_row[2];
    Ops::output_rows(t, idx, out_row);
    for (int st = 0; st < steps; ++st) {
        copy_wait<0>();
        // Every thread's copies of step st have landed, and every warp is past the products of
        // step st - 1, whose stage the next copies reuse: one barrier a step.
        __syncthreads();
        if (st + 1 < steps) {
            Ops::issue(t, c0, k0 + (st + 1) * kTileK, next_rows, vals, in, k, stage[(st + 1) & 1]);
            if (st + 2 < steps) Ops::input_rows(t, k0 + (st + 2) * kTileK, idx, next_rows);
        }
        Ops::compute(t, k0 + st * kTileK, stage[st & 1], acc);
    }
    Ops::store(t, c0, out_row, out, k, acc);
}

// The two stages live in dynamic shared memory (stage_bytes, above the 48 KB static limit).
template <int TC>
constexpr int stage_bytes() { return 2 * (int)sizeof(Stage<TC>); }

// A forward pass over right-hand sides that are zero outside the marked supernodes (a batch of
// source indicators: only a source's supernode and its ancestors receive anything): a tile of an
// unmarked node has a zero input block. Its update rows of a deterministic factor are written as
// zeros (the level's gather adds them), its Y rows too unless the backward pass is trimmed (and so
// does not read them: first_inner), and a tile that accumulates is skipped. Returns whether the tile was
// handled so.
__device__ __forceinline__ bool skip_inactive(const Tile& t, const unsigned char* active, int trimmed, int c0,
                                              int width, const int* idx, double* out, int k) {
    // A backward tile of an unmarked node is trimmed instead (first_inner); when the backward pass
    // trims, the Y rows of the forward diagonal tile, read by nothing else, are not written.
    if (active == nullptr || active[t.node] || t.tri == 2) return false;
    if (t.op == kAssign && (t.tri != 1 || !trimmed))
        for (int e = threadIdx.x; e < t.rows * width; e += blockDim.x) {
            const int i = e / width, c = c0 + e % width;
            if (c >= k) continue;
            const int r = t.out_rows < 0 ? t.out_base + t.r0 + i : idx[t.out_rows + t.r0 + i];
            out[(size_t)r * k + c] = 0.0;
        }
    return true;
}

// The first inner index a tile's product runs from. The backward tile of an unmarked node (its Y
// block zero: nothing reached it in the forward pass, which left its Y rows unwritten) starts past
// the Y block, at the node's off-diagonal rows.
__device__ __forceinline__ int first_inner(const Tile& t, const unsigned char* active) {
    return (active != nullptr && t.tri == 2 && !active[t.node]) ? max(t.k0, t.tri_k) : t.k0;
}

// One launch per phase: a CTA per (tile, column block of TC columns), the column block varying
// fastest, so a tile's blocks run side by side and its matrix block, read by each, comes from
// DRAM once (tile-major with the blocks apart, the second read missed L2: 757 against 619 MB a
// pass on the 131k torus at 64 columns in 32-column blocks).
template <int TC>
__global__ void __launch_bounds__(tile_threads<TC>(), TC == kTileCols ? kTileCtasPerSm : kTileCtasPerSmNarrow)
tile_product_kernel(const Tile* __restrict__ tiles, const double* __restrict__ vals,
                    const int* __restrict__ idx, double* rows, int k, const unsigned char* active, int trimmed) {
    extern __shared__ __align__(16) unsigned char shared_stages[];
    Stage<TC>* stage = reinterpret_cast<Stage<TC>*>(shared_stages);
    // The tile's fields in registers: read through a reference, the loop would load them again
    // from global memory after every barrier (0.420 -> 0.401 ms a pass on the 131k torus).
    const int blocks = (k + TC - 1) / TC;
    const Tile t = tiles[blockIdx.x / blocks];
    const int c0 = (int)(blockIdx.x % blocks) * TC;
    if (skip_inactive(t, active, trimmed, c0, TC, idx, rows, k)) return;
    tile_product<TC>(t, first_inner(t, active), c0, vals, idx, rows, rows, k, stage);
}

// The same tile product for a narrow batch (KP = 2, 4, 6 or 8 columns, the even stride of 1-8
// right-hand sides), where a 64-column tensor-core tile would compute 8-32 times the flops it
// needs: float64 FMAs in registers, the factor read once. A CTA per tile, 256 threads as (row,
// inner-dimension slice) pairs: thread (i, s) sums A(i, kk) in[kk] over kk = k0 + s, k0 + s + 4,
// ... for its KP columns, four steps at a time with every load of the four issued before their
// FMAs (the kernel is load-latency bound); the slices meet in shared memory and the first applies
// the tile's op.
constexpr int kNarrowThreads = 256;
constexpr int kNarrowSlices = kNarrowThreads / kTileRows;

template <int KP>
__global__ void __launch_bounds__(kNarrowThreads)
narrow_tile_kernel(const Tile* __restrict__ tiles, const double* __restrict__ vals,
                   const int* __restrict__ idx, double* rows, const unsigned char* active, int trimmed) {
    if (skip_inactive(tiles[blockIdx.x], active, trimmed, 0, KP, idx, rows, KP)) return;
    const double* in = rows;
    double* out = rows;
    __shared__ double other[kNarrowSlices - 1][kTileRows][KP];
    const Tile t = tiles[blockIdx.x];
    const int i = threadIdx.x % kTileRows, slice = threadIdx.x / kTileRows;
    double acc[KP];
#pragma unroll
    for (int c = 0; c < KP; ++c) acc[c] = 0.0;
    if (i < t.rows) {
        const double* M = vals + t.m;
        auto value = [&](int kk) {
            return t.trans ? __ldcg(M + (size_t)kk * t.ld + t.r0 + i) : __ldg(M + (size_t)(t.r0 + i) * t.ld + kk);
        };
        auto row = [&](int kk) { return t.in_rows < 0 ? t.in_base + kk : __ldg(idx + t.in_rows + kk); };
        auto add = [&](double a, int r) {
            const double2* x = reinterpret_cast<const double2*>(in + (size_t)r * KP);
#pragma unroll
            for (int c = 0; c < KP / 2; ++c) {
                const double2 v = __ldcg(x + c);
                acc[2 * c] = fma(a, v.x, acc[2 * c]);
                acc[2 * c + 1] = fma(a, v.y, acc[2 * c + 1]);
            }
        };
        if (t.trans) {
            // Column-major reads: the 64 threads of a slice read 64 consecutive values. Values a
            // thread alone reads go through L2 only (`__ldcg`): caching them in L1 measured slower.
            constexpr int kStep = kNarrowSlices;
            int kk = first_inner(t, active) + slice;
            for (; kk + 3 * kStep < t.k1; kk += 4 * kStep) {
                const int r0 = row(kk), r1 = row(kk + kStep), r2 = row(kk + 2 * kStep), r3 = row(kk + 3 * kStep);
                const double a0 = value(kk), a1 = value(kk + kStep), a2 = value(kk + 2 * kStep),
                             a3 = value(kk + 3 * kStep);
                add(a0, r0);
                add(a1, r1);
                add(a2, r2);
                add(a3, r3);
            }
            for (; kk < t.k1; kk += kStep) add(value(kk), row(kk));
        } else {
            // Row-major reads: a thread reads four consecutive values of its row as two 16-byte
            // loads (every block row starts on 16 bytes and k0 is even), slice s taking elements
            // 4 s .. 4 s + 3 of every 16; the one group that straddles k1 is read element by
            // element by its slice.
            constexpr int kGroup = 4 * kNarrowSlices;
            int kk = t.k0 + 4 * slice;
            for (; kk + 3 < t.k1; kk += kGroup) {
                const double2* p = reinterpret_cast<const double2*>(M + (size_t)(t.r0 + i) * t.ld + kk);
                const int r0 = row(kk), r1 = row(kk + 1), r2 = row(kk + 2), r3 = row(kk + 3);
                const double2 v01 = __ldcg(p), v23 = __ldcg(p + 1);
                add(v01.x, r0);
                add(v01.y, r1);
                add(v23.x, r2);
                add(v23.y, r3);
            }
            for (; kk < t.k1; ++kk) add(value(kk), row(kk));  // kk + 3 >= k1: at most 3
        }
    }
    if (slice > 0) {
#pragma unroll
        for (int c = 0; c < KP; ++c) other[slice - 1][i][c] = acc[c];
    }
    __syncthreads();
    if (slice > 0 || i >= t.rows) return;
    const int r = t.out_rows < 0 ? t.out_base + t.r0 + i : idx[t.out_rows + t.r0 + i];
    double* o = out + (size_t)r * KP;
#pragma unroll
    for (int c = 0; c < KP; ++c) {
        double v = acc[c];
#pragma unroll
        for (int s2 = 0; s2 < kNarrowSlices - 1; ++s2) v += other[s2][i][c];
        switch (t.op) {
            case kAssign: o[c] = v; break;
            case kAtomicSub: atomicAdd(o + c, -v); break;
            case kSub: o[c] = __ldcg(o + c) - v; break;
            default: atomicAdd(o + c, v); break;
        }
    }
}

// Zeroes rows [start, start + count) of y and x for every listed range (the outputs that split
// tiles accumulate into atomically).
__global__ void zero_rows_kernel(const int2* __restrict__ ranges, int n_ranges, int k,
                                 double* __restrict__ y, double* __restrict__ x) {
    const int2 range = ranges[blockIdx.x];
    const long long begin = (long long)range.x * k, end = (long long)(range.x + range.y) * k;
    for (long long t = begin + threadIdx.x; t < end; t += blockDim.x) {
        y[t] = 0.0;
        x[t] = 0.0;
    }
    (void)n_ranges;
}

// The deterministic forward update's gather: B[rows[t]] += the update rows src[offsets[t] ..
// offsets[t + 1]) in that order (a warp a target row, its lanes the columns).
__global__ void gather_updates_kernel(const int* __restrict__ offsets, const int* __restrict__ rows,
                                      const int* __restrict__ src, int n_targets, int k, double* work) {
    const int t = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (t >= n_targets) return;
    const int lane = threadIdx.x & 31;
    double* out = work + (size_t)rows[t] * k;
    for (int c = lane; c < k; c += 32) {
        double acc = out[c];
        for (int j = offsets[t]; j < offsets[t + 1]; ++j) acc += work[(size_t)src[j] * k + c];
        out[c] = acc;
    }
}

// Gathers rows of x (old numbering, k columns) into the factor's numbering at the even internal
// stride kp (a pad column is zero), zeroing pinned rows; or scatters back.
__global__ void permute_in_kernel(int n, int k, int kp, const int* __restrict__ perm,
                                  const char* __restrict__ pinned, const double* __restrict__ src,
                                  double* __restrict__ dst) {
    const long long total = (long long)n * kp;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / kp), c = (int)(t % kp);
        dst[t] = (pinned[i] || c >= k) ? 0.0 : src[(size_t)perm[i] * k + c];
    }
}

__global__ void permute_out_kernel(int n, int k, int kp, const int* __restrict__ perm,
                                   const double* __restrict__ src, double* __restrict__ dst,
                                   int accumulate, double scale) {
    const long long total = (long long)n * k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / k), c = (int)(t % k);
        double* d = dst + (size_t)perm[i] * k + c;
        const double v = scale * src[(size_t)i * kp + c];
        *d = accumulate ? *d + v : v;
    }
}

// r = b - A x over n_columns interleaved columns (float64).
__global__ void residual_kernel(int n, int k, const int* __restrict__ offsets,
                                const int* __restrict__ columns, const double* __restrict__ values,
                                const double* __restrict__ b, const double* __restrict__ x,
                                double* __restrict__ r) {
    const long long total = (long long)n * k;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(t / k), c = (int)(t % k);
        double acc = 0.0;
        for (int j = offsets[row]; j < offsets[row + 1]; ++j)
            acc = fma(values[j], x[(size_t)columns[j] * k + c], acc);
        r[t] = b[t] - acc;
    }
}

struct Factor {
    const Analysis* analysis = nullptr;
    int n = 0;
    bool singular = false;
    double sign = 1.0;       // the factor is of sign * A: solves scale its answers by sign
    double* vals = nullptr;  // device: all inverses and panels
    int* idx = nullptr;      // device: off-diagonal row lists
    int* perm = nullptr;     // device: new -> old
    int* iperm = nullptr;    // device: old -> new
    char* pinned = nullptr;  // device
    long long n_vals = 0;
    // Tile lists per (direction, level): host copies of counts, device tile arrays. Tiles name
    // rows of a work set's stacked [B; Y; X] buffer (B rows 0..n-1, Y rows n.., X rows 2n..).
    std::vector<Tile*> fwd, bwd;
    std::vector<int> n_fwd, n_bwd;
    int launches_per_pass = 0;
    std::vector<void*> owned;
    std::vector<void*> tile_owned;  // the tile lists and zero ranges (rebuilt by build_tiles)
    int2* zero = nullptr;  // row ranges split tiles accumulate into (zeroed each pass)
    int n_zero = 0;
    int tile_chunk = 0, tile_waves = 0;  // the split parameters the tile lists were built with
    // Column width of each level's tiles a direction (kTileCols or kTileColsNarrow): levels with
    // fewer tiles than narrow_waves waves of the resident grid take the narrow form (0: none; the
    // default, 64, every level: on the 131k torus at 64 columns 0.375 against 0.401 ms a pass).
    int narrow_waves = 64;
    std::vector<int> fwd_cols, bwd_cols;
    // Deterministic passes: no split tiles, and each node's forward update G B[own] written to its
    // own rows U of the work buffer (rows 3n ..), then added into its target rows by one gather a
    // level, every target row's contributions in node order -- no atomics anywhere in a pass.
    bool deterministic = false;
    long long n_update_rows = 0;               // rows of U (every node's off-diagonal rows)
    std::vector<int*> gather_offsets;          // per level: device CSR over its target rows
    std::vector<int*> gather_rows, gather_src;
    std::vector<int> n_gather;                 // per level: target rows
    // Device: each row's supernode and each supernode's parent (-1 at a root), for marking the
    // supernodes a batch of source indicators reaches.
    int* node_of_row = nullptr;
    int* parent_node = nullptr;
    int n_nodes = 0;
    // Per node: offsets of its [L11^-1; G] block in vals, of its row lists in idx, and its ld.
    std::vector<long long> inv_at, off_at;
    std::vector<int> rows_at, back_at, ld_at;
    size_t bytes = 0;
    // Recorded solve graphs, keyed by (columns, refinement steps, operator arrays).
    struct Recorded {
        int k, refine;
        const int *offsets, *columns;
        const double* values;
        cudaGraphExec_t exec;
        int launches;
    };
    // A set of work buffers sized for `cap_k` columns: B, Y, X in the factor's numbering (three
    // consecutive n-row blocks of one allocation, BYX), R the residual, RHS / SOL the caller's
    // right-hand side and solution copied in / out (old numbering), and the solve graphs recorded
    // over them. Passes on different sets are independent and may run concurrently (each set on
    // one stream at a time).
    struct WorkSet {
        int cap_k = 0;
        long long rows = 0;  // rows of the BYX allocation (3 n, plus U in a deterministic factor)
        double *BYX = nullptr, *R = nullptr, *RHS = nullptr, *SOL = nullptr;
        unsigned char* active = nullptr;  // device, one flag a supernode (marked sources)
        // B, Y and X at the even column stride kp of a call: n rows of kp doubles each.
        double* B() const { return BYX; }
        double* Y(int kp, int n) const { return BYX + (size_t)n * kp; }
        double* X(int kp, int n) const { return BYX + 2 * (size_t)n * kp; }
        // Bumped whenever the buffers are reallocated: a graph recorded outside the factor (over
        // ob_chol_work's pointers) is stale once it changes.
        long long generation = 0;
        std::vector<Recorded> graphs;
    };
    WorkSet sets[kWorkSets];
    cudaStream_t capture = nullptr;
};

int dev_alloc(Factor* F, void** p, size_t bytes, cudaStream_t stream) {
    OB_CUDA(pool_malloc(p, std::max<size_t>(bytes, 8), stream));
    F->owned.push_back(*p);
    F->bytes += bytes;
    return OB_OK;
}

int tile_alloc(Factor* F, void** p, size_t bytes, cudaStream_t stream) {
    OB_CUDA(pool_malloc(p, std::max<size_t>(bytes, 8), stream));
    F->tile_owned.push_back(*p);
    return OB_OK;
}

void factor_release(Factor* F) {
    if (F == nullptr) return;
    {
        std::lock_guard<std::recursive_mutex> guard(capture_mutex());
        cudaDeviceSynchronize();
    }
    for (auto& W : F->sets)
        for (auto& g : W.graphs) cudaGraphExecDestroy(g.exec);
    if (F->capture) cudaStreamDestroy(F->capture);
    for (void* p : F->owned) cudaFree(p);
    for (void* p : F->tile_owned) cudaFree(p);
    delete F;
}

// Lets the product kernels take their kStageBytes of dynamic shared memory (once per device).
int allow_stage_memory() {
    static int allowed[64] = {};
    int device = 0;
    OB_CUDA(cudaGetDevice(&device));
    if (device >= 0 && device < 64 && allowed[device]) return OB_OK;
    OB_CUDA(cudaFuncSetAttribute(tile_product_kernel<kTileCols>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 stage_bytes<kTileCols>()));
    OB_CUDA(cudaFuncSetAttribute(tile_product_kernel<kTileCols>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared));
    OB_CUDA(cudaFuncSetAttribute(tile_product_kernel<kTileColsNarrow>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, stage_bytes<kTileColsNarrow>()));
    OB_CUDA(cudaFuncSetAttribute(tile_product_kernel<kTileColsNarrow>,
                                 cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
    OB_CUDA(cudaFuncSetAttribute(tile_product_kernel<kTileColsSixteen>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, stage_bytes<kTileColsSixteen>()));
    OB_CUDA(cudaFuncSetAttribute(tile_product_kernel<kTileColsSixteen>,
                                 cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
    if (device >= 0 && device < 64) allowed[device] = 1;
    return OB_OK;
}

// The tile lists of the passes (and the row ranges their split tiles accumulate into), replacing
// any built before. chunk: the inner-dimension range of a split tile (0: never split); waves:
// levels with fewer tiles than that many waves of the resident grid (kTileCtasPerSm an SM) are split.
int build_tiles(Factor* F, int chunk, int waves, cudaStream_t stream) {
    for (void* p : F->tile_owned) OB_CUDA(cudaFreeAsync(p, stream));
    F->tile_owned.clear();
    F->zero = nullptr;
    F->n_zero = 0;
    F->gather_offsets.clear();
    F->gather_rows.clear();
    F->gather_src.clear();
    F->n_gather.clear();
    const int requested_chunk = chunk;
    if (F->deterministic) chunk = 0;  // split tiles accumulate atomically
    // One launch per tree level and direction. Forward at a level: every node's
    // Y[own] = L11^-1 B[own] and B[off rows] += G B[own] (atomic: siblings share ancestors' rows);
    // backward: X[own] = [L11^-1; G]^T [Y[own]; X[off rows]], one product over nc + noff. Each
    // reads only rows no tile of its launch writes. A level with few tiles has its long inner
    // dimensions split over several tiles (more CTAs, each a shorter latency-bound chain), which
    // then accumulate atomically into rows zeroed at the start of each pass; a level with `waves`
    // waves of tiles or more is not split.
    const Analysis& A = *F->analysis;
    const int ns = (int)A.nodes.size(), n = A.n;
    const std::vector<long long>&inv_at = F->inv_at, &off_at = F->off_at;
    const std::vector<int>&rows_at = F->rows_at, &back_at = F->back_at, &ld_at = F->ld_at;
    const int L = A.levels;
    const long long wave = (long long)kTileCtasPerSm * sm_count();
    auto tiles_of = [](int rows) { return (rows + kTileRows - 1) / kTileRows; };
    std::vector<long long> fwd_count(L, 0), bwd_count(L, 0);
    for (const Node& nd : A.nodes) {
        if (nd.count == 0) continue;
        fwd_count[nd.level] += tiles_of(nd.count) + tiles_of((int)nd.off_rows.size());
        bwd_count[nd.level] += tiles_of(nd.count);
    }
    auto emit = [chunk](std::vector<Tile>& list, Tile t, int K, bool may_split, int whole_op, int split_op) {
        const bool split = chunk > 0 && may_split && K > chunk + chunk / 2;
        for (int k0 = 0; k0 < K; k0 += split ? chunk : K) {
            t.k0 = k0;
            t.k1 = split ? std::min(K, k0 + chunk) : K;
            t.op = split ? split_op : whole_op;
            list.push_back(t);
        }
        return split;
    };
    std::vector<std::vector<Tile>> fw(L), bw(L);
    std::vector<int2> zero_ranges;
    // A deterministic factor's update rows: node s's at 3 n + u_at[s] .. + noff.
    std::vector<int> u_at(ns, 0);
    for (int s = 0, total = 0; s < ns; ++s) {
        u_at[s] = total;
        total += (int)A.nodes[s].off_rows.size();
    }
    for (int s = 0; s < ns; ++s) {
        const Node& nd = A.nodes[s];
        const int nc = nd.count, noff = (int)nd.off_rows.size(), ld = ld_at[s];
        if (nc == 0) continue;
        const bool split_fwd = fwd_count[nd.level] < waves * wave, split_bwd = bwd_count[nd.level] < waves * wave;
        bool zero = false;
        for (int r0 = 0; r0 < nc; r0 += kTileRows) {
            const int rows = std::min(kTileRows, nc - r0);
            // Forward diagonal: Y[own] = L11^-1 B[own].
            zero |= emit(fw[nd.level], Tile{inv_at[s], ld, 0, r0, rows, 0, 0, nd.start, -1, n + nd.start, -1, 0, 1, nc, s},
                         nc, split_fwd, kAssign, kAtomicAdd);
            // Backward: X[own] = [L11^-1; G]^T [Y[own]; X[off rows]].
            zero |= emit(bw[nd.level], Tile{inv_at[s], ld, 1, r0, rows, 0, 0, 0, back_at[s], 2 * n + nd.start, -1, 0, 2, nc, s},
                         nc + noff, split_bwd, kAssign, kAtomicAdd);
        }
        if (zero) zero_ranges.push_back(make_int2(nd.start, nc));
        for (int r0 = 0; r0 < noff; r0 += kTileRows) {
            const int rows = std::min(kTileRows, noff - r0);
            if (F->deterministic) {
                // Forward update: U[node] = G B[own], added into B[off rows] by the level's gather.
                emit(fw[nd.level], Tile{off_at[s], ld, 0, r0, rows, 0, 0, nd.start, -1, 3 * n + u_at[s], -1, 0, 0, 0, s},
                     nc, false, kAssign, kAssign);
                continue;
            }
            // Forward update: B[off rows] += G B[own].
            emit(fw[nd.level], Tile{off_at[s], ld, 0, r0, rows, 0, 0, nd.start, -1, 0, rows_at[s], 0, 0, 0, s},
                 nc, split_fwd, kAtomicAdd, kAtomicAdd);
        }
    }
    if (F->deterministic) {
        // Per level, every target row's update rows (U rows 3n + u_at[s] + r), nodes in index
        // order: the gather adds them in that order.
        std::vector<std::vector<std::pair<int, int>>> targets(L);
        for (int s = 0; s < ns; ++s) {
            const Node& nd = A.nodes[s];
            if (nd.count == 0) continue;
            for (int r = 0; r < (int)nd.off_rows.size(); ++r)
                targets[nd.level].push_back({nd.off_rows[r], 3 * n + u_at[s] + r});
        }
        F->gather_offsets.assign(L, nullptr);
        F->gather_rows.assign(L, nullptr);
        F->gather_src.assign(L, nullptr);
        F->n_gather.assign(L, 0);
        for (int l = 0; l < L; ++l) {
            auto& list = targets[l];
            if (list.empty()) continue;
            std::stable_sort(list.begin(), list.end(),
                             [](const std::pair<int, int>& a, const std::pair<int, int>& b) { return a.first < b.first; });
            std::vector<int> offsets, rows, src;
            for (size_t i = 0; i < list.size(); ++i) {
                if (i == 0 || list[i].first != list[i - 1].first) {
                    offsets.push_back((int)i);
                    rows.push_back(list[i].first);
                }
                src.push_back(list[i].second);
            }
            offsets.push_back((int)list.size());
            F->n_gather[l] = (int)rows.size();
            for (auto* vec : {&offsets, &rows, &src}) {
                int* d = nullptr;
                int st2 = tile_alloc(F, (void**)&d, sizeof(int) * vec->size(), stream);
                if (st2) return st2;
                OB_CUDA(cudaMemcpyAsync(d, vec->data(), sizeof(int) * vec->size(), cudaMemcpyHostToDevice, stream));
                (vec == &offsets ? F->gather_offsets : vec == &rows ? F->gather_rows : F->gather_src)[l] = d;
            }
            OB_CUDA(cudaStreamSynchronize(stream));  // the host lists go out of scope
        }
    }
    // Adjacent ranges joined, then cut into pieces of at most 16 rows: one block each, so the
    // zeroing launch is balanced however large a merged node is.
    std::vector<int2> pieces;
    for (size_t i = 0; i < zero_ranges.size();) {
        int2 r = zero_ranges[i++];
        while (i < zero_ranges.size() && zero_ranges[i].x == r.x + r.y) r.y += zero_ranges[i++].y;
        for (int o = 0; o < r.y; o += 16) pieces.push_back(make_int2(r.x + o, std::min(16, r.y - o)));
    }
    zero_ranges.swap(pieces);
    F->n_zero = (int)zero_ranges.size();
    int st = OB_OK;
    if (F->n_zero > 0) {
        st = tile_alloc(F, (void**)&F->zero, sizeof(int2) * zero_ranges.size(), stream);
        if (st) return st;
        OB_CUDA(cudaMemcpyAsync(F->zero, zero_ranges.data(), sizeof(int2) * zero_ranges.size(),
                                cudaMemcpyHostToDevice, stream));
    }
    auto push = [&](std::vector<std::vector<Tile>>& lists, std::vector<Tile*>& dst,
                    std::vector<int>& counts) -> int {
        dst.assign(L, nullptr);
        counts.assign(L, 0);
        for (int l = 0; l < L; ++l) {
            counts[l] = (int)lists[l].size();
            if (lists[l].empty()) continue;
            int st2 = tile_alloc(F, (void**)&dst[l], sizeof(Tile) * lists[l].size(), stream);
            if (st2) return st2;
            OB_CUDA(cudaMemcpyAsync(dst[l], lists[l].data(), sizeof(Tile) * lists[l].size(),
                                    cudaMemcpyHostToDevice, stream));
        }
        return OB_OK;
    };
    st = push(fw, F->fwd, F->n_fwd);
    if (!st) st = push(bw, F->bwd, F->n_bwd);
    if (st) return st;
    F->fwd_cols.assign(L, kTileCols);
    F->bwd_cols.assign(L, kTileCols);
    for (int l = 0; l < L; ++l) {
        if (F->n_fwd[l] < (long long)F->narrow_waves * wave) F->fwd_cols[l] = kTileColsNarrow;
        if (F->n_bwd[l] < (long long)F->narrow_waves * wave) F->bwd_cols[l] = kTileColsNarrow;
    }
    F->launches_per_pass = 0;
    for (int l = 0; l < L; ++l)
        F->launches_per_pass += (F->n_fwd[l] > 0) + (F->n_bwd[l] > 0) + (F->deterministic && F->n_gather[l] > 0);
    OB_CUDA(cudaStreamSynchronize(stream));  // host staging buffers go out of scope
    F->tile_chunk = requested_chunk;
    F->tile_waves = waves;
    return OB_OK;
}

// The device factor: its block layout and row lists (from the analysis), then the numeric
// factorisation of sign * values on the device (device_factor, ob_chol_factor.cu), then the
// passes' tile lists.
int setup_factor(Factor* F, const double* values, double sign, int pin_mode, cudaStream_t stream) {
    if (int st0 = allow_stage_memory()) return st0;
    Analysis& A = *const_cast<Analysis*>(F->analysis);
    const int ns = (int)A.nodes.size();
    const int n = A.n;
    // Per node the stored block is [L11^-1; G] (nc + noff rows, G = -L21 L11^-1), every block row
    // padded to a multiple of 8 doubles (and every block starting on one), so the tile kernel's
    // 16-byte asynchronous copies are always aligned. idx holds per node its off-diagonal rows
    // (B rows, the forward update's outputs) and the backward product's input rows: its own Y rows
    // then its off-diagonal X rows, in the stacked [B; Y; X] numbering.
    BlockLayout layout = block_layout(A);
    OB_REQUIRE(layout.total_rows < (1LL << 31) && 3LL * n < (1LL << 31), "ob_chol_factor: factor too large");
    std::vector<int> idx(std::max<long long>(layout.total_rows, 1));
    for (int s = 0; s < ns; ++s) {
        const Node& nd = A.nodes[s];
        const int nc = nd.count, noff = (int)nd.off_rows.size();
        std::copy(nd.off_rows.begin(), nd.off_rows.end(), idx.begin() + layout.rows_at[s]);
        for (int i = 0; i < nc; ++i) idx[layout.back_at[s] + i] = n + nd.start + i;
        for (int r = 0; r < noff; ++r) idx[layout.back_at[s] + nc + r] = 2 * n + nd.off_rows[r];
    }
    F->n_vals = layout.total;
    int st = dev_alloc(F, (void**)&F->vals, sizeof(double) * std::max<long long>(layout.total, 1), stream);
    if (!st) st = dev_alloc(F, (void**)&F->idx, sizeof(int) * idx.size(), stream);
    if (!st) st = dev_alloc(F, (void**)&F->perm, sizeof(int) * A.n, stream);
    if (!st) st = dev_alloc(F, (void**)&F->iperm, sizeof(int) * A.n, stream);
    if (!st) st = dev_alloc(F, (void**)&F->pinned, std::max(A.n, 1), stream);
    if (st) return st;
    OB_CUDA(cudaMemcpyAsync(F->idx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice,
                            stream));
    OB_CUDA(cudaMemcpyAsync(F->iperm, A.iperm.data(), sizeof(int) * A.n, cudaMemcpyHostToDevice,
                            stream));
    OB_CUDA(cudaMemcpyAsync(F->perm, A.perm.data(), sizeof(int) * A.n, cudaMemcpyHostToDevice,
                            stream));
    // Each row's supernode and each supernode's parent, and a marking buffer per work set.
    std::vector<int> node_of_row(std::max(n, 1), -1), parent(std::max(ns, 1), -1);
    for (int s = 0; s < ns; ++s) {
        parent[s] = A.nodes[s].parent;
        for (int j = 0; j < A.nodes[s].count; ++j) node_of_row[A.nodes[s].start + j] = s;
    }
    if ((st = dev_alloc(F, (void**)&F->node_of_row, sizeof(int) * node_of_row.size(), stream)) ||
        (st = dev_alloc(F, (void**)&F->parent_node, sizeof(int) * parent.size(), stream)))
        return st;
    OB_CUDA(cudaMemcpyAsync(F->node_of_row, node_of_row.data(), sizeof(int) * node_of_row.size(),
                            cudaMemcpyHostToDevice, stream));
    OB_CUDA(cudaMemcpyAsync(F->parent_node, parent.data(), sizeof(int) * parent.size(),
                            cudaMemcpyHostToDevice, stream));
    F->n_nodes = ns;
    for (auto& W : F->sets)
        if ((st = dev_alloc(F, (void**)&W.active, std::max(ns, 1), stream))) return st;
    long long update_rows = 0;
    for (const Node& nd : A.nodes) update_rows += (long long)nd.off_rows.size();
    F->n_update_rows = update_rows;
    F->inv_at = std::move(layout.inv_at);
    F->off_at = std::move(layout.off_at);
    F->rows_at = std::move(layout.rows_at);
    F->back_at = std::move(layout.back_at);
    F->ld_at = std::move(layout.ld_at);
    // The numeric factorisation (synchronises once, to read its pivot status).
    if ((st = device_factor(A, values, sign, pin_mode, F->vals, F->pinned, stream))) return st;
    if ((st = build_tiles(F, kSplitK, 2, stream))) return st;
    OB_CUDA(cudaStreamSynchronize(stream));  // host staging buffers go out of scope
    return OB_OK;
}

// The internal column stride of B, Y and X: even, so every row starts on 16 bytes.
inline int even_columns(int k) { return (k + 1) & ~1; }

int ensure_work(Factor* F, Factor::WorkSet& W, int k, cudaStream_t stream) {
    const long long rows = 3LL * F->n + (F->deterministic ? F->n_update_rows : 0);
    if (k <= W.cap_k && rows == W.rows) return OB_OK;
    if (W.cap_k > k) k = W.cap_k;  // a change of rows keeps the widest width
    // Growing the buffers invalidates every recorded graph (they name the old ones).
    OB_CUDA(cudaStreamSynchronize(stream));
    for (auto& g : W.graphs) cudaGraphExecDestroy(g.exec);
    W.graphs.clear();
    // The smaller buffers go (no graph names them any more): one set at the widest width.
    const size_t old_row = sizeof(double) * (size_t)(W.cap_k > 0 ? even_columns(W.cap_k) : 0);
    for (double** p : {&W.BYX, &W.R, &W.RHS, &W.SOL}) {
        if (*p == nullptr) continue;
        auto it = std::find(F->owned.begin(), F->owned.end(), (void*)*p);
        if (it != F->owned.end()) {
            F->owned.erase(it);
            F->bytes -= old_row * (size_t)(p == &W.BYX ? W.rows : F->n);
            OB_CUDA(cudaFreeAsync(*p, stream));
        }
        *p = nullptr;
    }
    const size_t row = sizeof(double) * (size_t)even_columns(k);
    for (double** p : {&W.BYX, &W.R, &W.RHS, &W.SOL}) {
        int st = dev_alloc(F, (void**)p, row * (size_t)(p == &W.BYX ? rows : F->n), stream);
        if (st) return st;
    }
    W.rows = rows;
    W.cap_k = k;
    ++W.generation;
    return OB_OK;
}

// x_new = A^-1 b_new in the factor's numbering (B is consumed); k is the even internal stride.
// Marks the supernodes a batch of source indicators reaches: each source's supernode (through
// the factor's numbering) and every ancestor, up to one already marked (whose marker goes on to
// the root). sources[source_offsets[0] .. source_offsets[n_columns]) are vertex indices, a thread
// a source over the grid (the walks run side by side: two that meet both write 1, and one that
// stops at a marked node leaves the rest of the chain to the thread that marked it).
constexpr int kMarkBlocks = 32;
__global__ void mark_sources_kernel(const int* __restrict__ sources, const int* __restrict__ source_offsets,
                                    int n_columns, const int* __restrict__ iperm, const int* __restrict__ node_of_row,
                                    const int* __restrict__ parent, unsigned char* active) {
    const int total = source_offsets[n_columns] - source_offsets[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        int node = node_of_row[iperm[sources[source_offsets[0] + i]]];
        while (node >= 0) {
            const unsigned char was = active[node];
            active[node] = 1;
            if (was) break;
            node = parent[node];
        }
    }
}

// forward_active: the marked supernodes of a batch of source indicators (see skip_inactive and
// first_inner), or nullptr.
int triangular_solves(Factor* F, Factor::WorkSet& W, int k, cudaStream_t stream,
                      const unsigned char* forward_active = nullptr) {
    const int L = F->analysis->levels;
    // The tiles address rows up to 3 n (plus the update rows of a deterministic factor): the work
    // buffer must have been allocated for the factor's present mode.
    OB_REQUIRE(W.BYX != nullptr && W.rows == 3LL * F->n + (F->deterministic ? F->n_update_rows : 0) &&
                   k <= even_columns(W.cap_k),
               "chol pass: work buffers not prepared for %d columns in this mode", k);
    if (F->n_zero > 0) {
        zero_rows_kernel<<<F->n_zero, 256, 0, stream>>>(F->zero, F->n_zero, k, W.Y(k, F->n), W.X(k, F->n));
        OB_CHECK_LAUNCH("chol zero split rows");
    }
    // A level's launch: the float64 tensor-core tiles, or for a narrow batch (stride 2-8) the
    // register kernel, which does not compute a 64-column tile's idle columns.
    // The backward pass is trimmed past the zero Y blocks of unmarked nodes, except in a
    // deterministic factor: there a query's sums must not depend on the marks other queries of its
    // batch add (trimming changes how the tensor-core steps group the inner dimension).
    const int trimmed = forward_active != nullptr && !F->deterministic;
    auto level = [&](const Tile* tiles, int count, int cols, const unsigned char* active, const char* what) {
        switch (k) {
            case 2: narrow_tile_kernel<2><<<count, kNarrowThreads, 0, stream>>>(tiles, F->vals, F->idx, W.BYX, active, trimmed); break;
            case 4: narrow_tile_kernel<4><<<count, kNarrowThreads, 0, stream>>>(tiles, F->vals, F->idx, W.BYX, active, trimmed); break;
            case 6: narrow_tile_kernel<6><<<count, kNarrowThreads, 0, stream>>>(tiles, F->vals, F->idx, W.BYX, active, trimmed); break;
            case 8: narrow_tile_kernel<8><<<count, kNarrowThreads, 0, stream>>>(tiles, F->vals, F->idx, W.BYX, active, trimmed); break;
            default:
                if (k <= kTileColsSixteen)
                    tile_product_kernel<kTileColsSixteen>
                        <<<(unsigned)count, tile_threads<kTileColsSixteen>(), stage_bytes<kTileColsSixteen>(),
                           stream>>>(tiles, F->vals, F->idx, W.BYX, k, active, trimmed);
                else if (cols == kTileColsNarrow)
                    tile_product_kernel<kTileColsNarrow>
                        <<<(unsigned)count * ceil_div(k, kTileColsNarrow), tile_threads<kTileColsNarrow>(),
                           stage_bytes<kTileColsNarrow>(),
                           stream>>>(tiles, F->vals, F->idx, W.BYX, k, active, trimmed);
                else
                    tile_product_kernel<kTileCols><<<(unsigned)count * ceil_div(k, kTileCols), tile_threads<kTileCols>(),
                                                      stage_bytes<kTileCols>(), stream>>>(tiles, F->vals, F->idx,
                                                                                          W.BYX, k, active, trimmed);
        }
        OB_CHECK_LAUNCH(what);
        return OB_OK;
    };
    int st = OB_OK;
    for (int l = 0; l < L && st == OB_OK; ++l) {
        if (F->n_fwd[l]) st = level(F->fwd[l], F->n_fwd[l], F->fwd_cols[l], forward_active, "chol forward level");
        if (st == OB_OK && F->deterministic && F->n_gather[l] > 0) {
            gather_updates_kernel<<<ceil_div(F->n_gather[l], 8), 256, 0, stream>>>(
                F->gather_offsets[l], F->gather_rows[l], F->gather_src[l], F->n_gather[l], k, W.BYX);
            OB_CHECK_LAUNCH("chol deterministic gather");
        }
    }
    // The backward pass starts past the zero Y block of every node the forward pass left unmarked.
    for (int l = L - 1; l >= 0 && st == OB_OK; --l)
        if (F->n_bwd[l])
            st = level(F->bwd[l], F->n_bwd[l], F->bwd_cols[l], trimmed ? forward_active : nullptr, "chol backward level");
    return st;
}

int grid_for(long long total) {
    return (int)std::max(1LL, std::min((total + 255) / 256, (long long)8 * sm_count()));
}

// The whole solve on the factor's own buffers: SOL = A^-1 RHS plus `refine` refinement steps.
int enqueue_solve(Factor* F, Factor::WorkSet& W, int k, int refine, const int* offsets, const int* columns,
                  const double* values, cudaStream_t stream) {
    const int n = F->n, kp = even_columns(k);
    const int grid = grid_for((long long)n * kp);
    permute_in_kernel<<<grid, 256, 0, stream>>>(n, k, kp, F->perm, F->pinned, W.RHS, W.B());
    OB_CHECK_LAUNCH("chol permute in");
    int st = triangular_solves(F, W, kp, stream);
    if (st) return st;
    permute_out_kernel<<<grid, 256, 0, stream>>>(n, k, kp, F->perm, W.X(kp, n), W.SOL, 0, F->sign);
    OB_CHECK_LAUNCH("chol permute out");
    // Iterative refinement in float64: x += A^-1 (b - A x).
    for (int it = 0; it < refine; ++it) {
        residual_kernel<<<grid, 256, 0, stream>>>(n, k, offsets, columns, values, W.RHS, W.SOL,
                                                  W.R);
        OB_CHECK_LAUNCH("chol residual");
        permute_in_kernel<<<grid, 256, 0, stream>>>(n, k, kp, F->perm, F->pinned, W.R, W.B());
        OB_CHECK_LAUNCH("chol permute in");
        st = triangular_solves(F, W, kp, stream);
        if (st) return st;
        permute_out_kernel<<<grid, 256, 0, stream>>>(n, k, kp, F->perm, W.X(kp, n), W.SOL, 1, F->sign);
        OB_CHECK_LAUNCH("chol permute out");
    }
    return OB_OK;
}

// The recorded graph of enqueue_solve for (k, refine, operator), recorded on first use.
int solve_graph(Factor* F, Factor::WorkSet& W, int k, int refine, const int* offsets, const int* columns,
                const double* values, Factor::Recorded** out) {
    for (auto& g : W.graphs)
        if (g.k == k && g.refine == refine && g.offsets == offsets && g.columns == columns &&
            g.values == values) {
            *out = &g;
            return OB_OK;
        }
    if (F->capture == nullptr) OB_CUDA(cudaStreamCreateWithFlags(&F->capture, cudaStreamNonBlocking));
    // Launches are counted at each replay (the graph's kernel nodes), not at capture.
    std::lock_guard<std::recursive_mutex> guard(capture_mutex());
    suppress_counting(1);
    cudaError_t e = cudaStreamBeginCapture(F->capture, cudaStreamCaptureModeThreadLocal);
    // refine < 0 records the bare triangular passes B -> X in the factor's own numbering.
    int st = e != cudaSuccess ? cuda_status(e, "ob_chol_solve: begin capture")
             : refine < 0     ? triangular_solves(F, W, even_columns(k), F->capture)
                              : enqueue_solve(F, W, k, refine, offsets, columns, values, F->capture);
    cudaGraph_t graph = nullptr;
    if (e == cudaSuccess) e = cudaStreamEndCapture(F->capture, &graph);
    suppress_counting(-1);
    cudaGraphExec_t exec = nullptr;
    size_t nodes = 0;
    if (st == OB_OK && e == cudaSuccess) {
        cudaGraphGetNodes(graph, nullptr, &nodes);
        e = cudaGraphInstantiate(&exec, graph, 0);
    }
    if (graph) cudaGraphDestroy(graph);
    if (st != OB_OK || e != cudaSuccess) {
        cudaGetLastError();
        return st != OB_OK ? st : cuda_status(e, "ob_chol_solve: capture");
    }
    W.graphs.push_back(Factor::Recorded{k, refine, offsets, columns, values, exec, (int)nodes});
    *out = &W.graphs.back();
    return OB_OK;
}


}  // namespace
}  // namespace ob

using namespace ob;

extern "C" {

int ob_chol_analyse(int n, const int32_t* offsets, const int32_t* columns, const float* xyz,
                    int leaf_size, void** analysis, ob_stream_t stream_) {
    return ob_chol_analyse_blocked(n, 1, offsets, columns, xyz, leaf_size, analysis, stream_);
}

int ob_chol_analyse_blocked(int n, int block, const int32_t* offsets, const int32_t* columns, const float* xyz,
                            int leaf_size, void** analysis, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(analysis != nullptr, "ob_chol_analyse: null output");
    *analysis = nullptr;
    OB_REQUIRE(n >= 1 && offsets && columns, "ob_chol_analyse: bad argument");
    OB_REQUIRE(block >= 1 && n % block == 0, "ob_chol_analyse_blocked: %d rows are not groups of %d", n, block);
    std::vector<int> off(n + 1);
    OB_CUDA(cudaMemcpyAsync(off.data(), offsets, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost,
                            stream));
    OB_CUDA(cudaStreamSynchronize(stream));
    std::vector<int> col(std::max(off[n], 1));
    std::vector<float> pts;
    OB_CUDA(cudaMemcpyAsync(col.data(), columns, sizeof(int) * off[n], cudaMemcpyDeviceToHost,
                            stream));
    if (xyz != nullptr) {
        pts.resize(3 * (size_t)(n / block));
        OB_CUDA(cudaMemcpyAsync(pts.data(), xyz, sizeof(float) * 3 * (size_t)(n / block),
                                cudaMemcpyDeviceToHost, stream));
    }
    OB_CUDA(cudaStreamSynchronize(stream));
    col.resize(off[n]);
    Analysis* A = new Analysis();
    int st = analyse(n, std::move(off), std::move(col), xyz ? pts.data() : nullptr, leaf_size, A, block);
    if (st) {
        delete A;
        return st;
    }
    *analysis = A;
    return OB_OK;
}

int ob_chol_host_analyse(int n, const int32_t* offsets, const int32_t* columns, const float* xyz,
                         int leaf_size, void** analysis) {
    OB_REQUIRE(analysis != nullptr && n >= 1 && offsets && columns, "ob_chol_host_analyse: bad argument");
    *analysis = nullptr;
    std::vector<int> off(offsets, offsets + n + 1), col(columns, columns + offsets[n]);
    Analysis* A = new Analysis();
    int st = analyse(n, std::move(off), std::move(col), xyz, leaf_size, A);
    if (st) {
        delete A;
        return st;
    }
    *analysis = A;
    return OB_OK;
}

int ob_chol_analysis_nodes(void* analysis, int32_t* out) {
    OB_REQUIRE(analysis && out, "ob_chol_analysis_nodes: bad argument");
    const Analysis* A = static_cast<Analysis*>(analysis);
    for (size_t s = 0; s < A->nodes.size(); ++s) {
        out[4 * s] = A->nodes[s].level;
        out[4 * s + 1] = A->nodes[s].count;
        out[4 * s + 2] = (int)A->nodes[s].off_rows.size();
        out[4 * s + 3] = A->nodes[s].parent;
    }
    return OB_OK;
}

int ob_chol_analysis_info(void* analysis, long long* info) {
    OB_REQUIRE(analysis && info, "ob_chol_analysis_info: bad argument");
    const Analysis* A = static_cast<Analysis*>(analysis);
    info[0] = A->n;
    info[1] = (long long)A->nodes.size();
    info[2] = A->levels;
    info[3] = A->factor_entries;
    long long widest = 0;
    for (const Node& nd : A->nodes) widest = std::max<long long>(widest, nd.count + nd.off_rows.size());
    info[4] = widest;
    return OB_OK;
}

int ob_chol_analysis_destroy(void* analysis) {
    delete static_cast<Analysis*>(analysis);
    return OB_OK;
}

int ob_chol_factor(void* analysis, const double* values, int singular, int negated, void** factor,
                   ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(analysis && values && factor, "ob_chol_factor: bad argument");
    OB_REQUIRE(singular >= kPinNone && singular <= kPinZeroSum, "ob_chol_factor: singular = %d outside [0, 2]",
               singular);
    *factor = nullptr;
    Analysis* A = static_cast<Analysis*>(analysis);
    Factor* F = new Factor();
    F->analysis = A;
    F->n = A->n;
    F->singular = singular != kPinNone;
    F->sign = negated ? -1.0 : 1.0;
    int st = setup_factor(F, values, F->sign, singular, stream);
    if (st) {
        factor_release(F);
        if (st == OB_ERR_INDEFINITE) return fail(OB_ERR_INDEFINITE, "ob_chol_factor: not positive definite");
        return st;
    }
    *factor = F;
    return OB_OK;
}

int ob_chol_solve(void* factor, const double* rhs, double* x, int n_columns, int refine,
                  const int32_t* offsets, const int32_t* columns, const double* values,
                  ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(factor && n_columns >= 1 && refine >= 0, "ob_chol_solve: bad argument");
    OB_REQUIRE(refine == 0 || (offsets && columns && values),
               "ob_chol_solve: refinement needs the operator");
    Factor* F = static_cast<Factor*>(factor);
    Factor::WorkSet& W = F->sets[0];
    int st = ensure_work(F, W, n_columns, stream);
    if (st) return st;
    const size_t bytes = sizeof(double) * (size_t)F->n * n_columns;
    if (rhs != nullptr && rhs != W.RHS)
        OB_CUDA(cudaMemcpyAsync(W.RHS, rhs, bytes, cudaMemcpyDeviceToDevice, stream));
    Factor::Recorded* g = nullptr;
    st = solve_graph(F, W, n_columns, refine, refine ? offsets : nullptr, refine ? columns : nullptr,
                     refine ? values : nullptr, &g);
    if (st) return st;
    OB_CUDA(cudaGraphLaunch(g->exec, stream));
    count_launch((uint64_t)g->launches);
    if (x != nullptr && x != W.SOL)
        OB_CUDA(cudaMemcpyAsync(x, W.SOL, bytes, cudaMemcpyDeviceToDevice, stream));
    return OB_OK;
}

int ob_chol_work(void* factor, int n_columns, double** rhs, double** solution, int* stride,
                 const int32_t** iperm, const char** pinned, ob_stream_t stream_) {
    return ob_chol_work_set(factor, 0, n_columns, rhs, solution, stride, iperm, pinned, stream_);
}

int ob_chol_work_set(void* factor, int set, int n_columns, double** rhs, double** solution, int* stride,
                     const int32_t** iperm, const char** pinned, ob_stream_t stream_) {
    OB_REQUIRE(factor && rhs && solution && stride && iperm && pinned && n_columns >= 1,
               "ob_chol_work: bad argument");
    OB_REQUIRE(set >= 0 && set < kWorkSets, "ob_chol_work: set %d outside [0, %d)", set, kWorkSets);
    Factor* F = static_cast<Factor*>(factor);
    Factor::WorkSet& W = F->sets[set];
    int st = ensure_work(F, W, n_columns, as_stream(stream_));
    if (st) return st;
    *rhs = W.B();
    *solution = W.X(even_columns(n_columns), F->n);
    *stride = even_columns(n_columns);
    *iperm = F->iperm;
    *pinned = F->pinned;
    return OB_OK;
}

int ob_chol_solve_in_place(void* factor, int n_columns, ob_stream_t stream_) {
    return ob_chol_solve_in_place_set(factor, 0, n_columns, stream_);
}

int ob_chol_solve_in_place_set(void* factor, int set, int n_columns, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(factor && n_columns >= 1, "ob_chol_solve_in_place: bad argument");
    OB_REQUIRE(set >= 0 && set < kWorkSets, "ob_chol_solve_in_place: set %d outside [0, %d)", set, kWorkSets);
    Factor* F = static_cast<Factor*>(factor);
    Factor::WorkSet& W = F->sets[set];
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    OB_CUDA(cudaStreamIsCapturing(stream, &capturing));
    if (capturing == cudaStreamCaptureStatusActive) {
        // Recorded into the caller's graph: the passes' kernels themselves (the buffers must
        // already hold n_columns: a capture cannot allocate them).
        OB_REQUIRE(n_columns <= W.cap_k, "ob_chol_solve_in_place: %d columns not prepared before "
                   "capture (ob_chol_work first)", n_columns);
        return triangular_solves(F, W, even_columns(n_columns), stream);
    }
    int st = ensure_work(F, W, n_columns, stream);
    if (st) return st;
    Factor::Recorded* g = nullptr;
    st = solve_graph(F, W, n_columns, -1, nullptr, nullptr, nullptr, &g);
    if (st) return st;
    OB_CUDA(cudaGraphLaunch(g->exec, stream));
    count_launch((uint64_t)g->launches);
    return OB_OK;
}

int ob_chol_solve_in_place_sources(void* factor, int set, int n_columns, const int32_t* sources,
                                   const int32_t* source_offsets, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(factor && n_columns >= 1 && sources && source_offsets, "ob_chol_solve_in_place_sources: bad argument");
    OB_REQUIRE(set >= 0 && set < kWorkSets, "ob_chol_solve_in_place_sources: set %d outside [0, %d)", set,
               kWorkSets);
    Factor* F = static_cast<Factor*>(factor);
    Factor::WorkSet& W = F->sets[set];
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    OB_CUDA(cudaStreamIsCapturing(stream, &capturing));
    if (capturing == cudaStreamCaptureStatusActive) {
        OB_REQUIRE(n_columns <= W.cap_k, "ob_chol_solve_in_place_sources: %d columns not prepared before "
                   "capture (ob_chol_work first)", n_columns);
    } else {
        int st = ensure_work(F, W, n_columns, stream);
        if (st) return st;
    }
    OB_CUDA(cudaMemsetAsync(W.active, 0, std::max(F->n_nodes, 1), stream));
    mark_sources_kernel<<<kMarkBlocks, 256, 0, stream>>>(sources, source_offsets, n_columns, F->iperm, F->node_of_row,
                                              F->parent_node, W.active);
    OB_CHECK_LAUNCH("chol mark sources");
    return triangular_solves(F, W, even_columns(n_columns), stream, W.active);
}

int ob_chol_buffers(void* factor, int n_columns, double** rhs, double** solution,
                    ob_stream_t stream_) {
    OB_REQUIRE(factor && rhs && solution && n_columns >= 1, "ob_chol_buffers: bad argument");
    Factor* F = static_cast<Factor*>(factor);
    Factor::WorkSet& W = F->sets[0];
    int st = ensure_work(F, W, n_columns, as_stream(stream_));
    if (st) return st;
    *rhs = W.RHS;
    *solution = W.SOL;
    return OB_OK;
}

int ob_chol_time_solve(void* factor, int n_columns, int reps, float* ms, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(factor && ms && reps >= 1 && n_columns >= 1, "ob_chol_time_solve: bad argument");
    Factor* F = static_cast<Factor*>(factor);
    Factor::WorkSet& W = F->sets[0];
    int st = ensure_work(F, W, n_columns, stream);
    if (st) return st;
    cudaEvent_t start, end;
    OB_CUDA(cudaEventCreate(&start));
    OB_CUDA(cudaEventCreate(&end));
    cudaEventRecord(start, stream);
    for (int i = 0; i < reps && st == OB_OK; ++i)
        st = triangular_solves(F, W, even_columns(n_columns), stream);
    cudaEventRecord(end, stream);
    cudaError_t e = cudaEventSynchronize(end);
    float total = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&total, start, end);
    cudaEventDestroy(start);
    cudaEventDestroy(end);
    if (st) return st;
    if (e != cudaSuccess) return cuda_status(e, "ob_chol_time_solve");
    *ms = total / (float)reps;
    return OB_OK;
}

int ob_chol_tile(void* factor, int chunk, int waves, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(factor != nullptr && waves >= 0 && waves <= 64, "ob_chol_tile: bad argument");
    // A split tile's inner range starts at a multiple of chunk, and the tile kernels read the
    // factor's rows from there in 16-byte pieces: chunk must keep every start on 16 bytes.
    OB_REQUIRE(chunk == 0 || (chunk >= 16 && chunk <= 4096 && chunk % 8 == 0),
               "ob_chol_tile: chunk %d is not 0 or a multiple of 8 in [16, 4096]", chunk);
    Factor* F = static_cast<Factor*>(factor);
    if (chunk == F->tile_chunk && waves == F->tile_waves) return OB_OK;
    {
        // No pass of this factor may be in flight while its tile lists are replaced.
        std::lock_guard<std::recursive_mutex> guard(capture_mutex());
        OB_CUDA(cudaDeviceSynchronize());
    }
    // Every recorded pass names the old lists: drop them, and move the work generations so the
    // callers' own recordings are made again.
    for (auto& W : F->sets) {
        for (auto& g : W.graphs) cudaGraphExecDestroy(g.exec);
        W.graphs.clear();
        ++W.generation;
    }
    return build_tiles(F, chunk, waves, stream);
}

int ob_chol_tile_columns(void* factor, int narrow_waves, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(factor != nullptr && narrow_waves >= 0 && narrow_waves <= 64, "ob_chol_tile_columns: bad argument");
    Factor* F = static_cast<Factor*>(factor);
    if (narrow_waves == F->narrow_waves) return OB_OK;
    {
        std::lock_guard<std::recursive_mutex> guard(capture_mutex());
        OB_CUDA(cudaDeviceSynchronize());
    }
    for (auto& W : F->sets) {
        for (auto& g : W.graphs) cudaGraphExecDestroy(g.exec);
        W.graphs.clear();
        ++W.generation;
    }
    F->narrow_waves = narrow_waves;
    return build_tiles(F, F->tile_chunk, F->tile_waves, stream);
}

int ob_chol_set_deterministic(void* factor, int on, ob_stream_t stream_) {
    cudaStream_t stream = as_stream(stream_);
    OB_REQUIRE(factor != nullptr, "ob_chol_set_deterministic: bad argument");
    Factor* F = static_cast<Factor*>(factor);
    if (F->deterministic == (on != 0)) return OB_OK;
    {
        // No pass of this factor may be in flight while its tiles and buffers are replaced.
        std::lock_guard<std::recursive_mutex> guard(capture_mutex());
        OB_CUDA(cudaDeviceSynchronize());
    }
    for (auto& W : F->sets) {
        for (auto& g : W.graphs) cudaGraphExecDestroy(g.exec);
        W.graphs.clear();
        ++W.generation;
    }
    F->deterministic = on != 0;
    int st = build_tiles(F, F->tile_chunk, F->tile_waves, stream);
    // Work buffers already made are remade at the new row count now (a recording made later
    // cannot allocate them).
    for (auto& W : F->sets)
        if (!st && W.cap_k > 0) st = ensure_work(F, W, W.cap_k, stream);
    if (!st) OB_CUDA(cudaStreamSynchronize(stream));
    return st;
}

int ob_chol_work_generation(void* factor, long long* generation) {
    return ob_chol_work_generation_set(factor, 0, generation);
}

int ob_chol_work_generation_set(void* factor, int set, long long* generation) {
    OB_REQUIRE(factor && generation && set >= 0 && set < kWorkSets, "ob_chol_work_generation: bad argument");
    *generation = static_cast<Factor*>(factor)->sets[set].generation;
    return OB_OK;
}

int ob_chol_info(void* factor, long long* info) {
    OB_REQUIRE(factor && info, "ob_chol_info: bad argument");
    Factor* F = static_cast<Factor*>(factor);
    info[0] = F->n;
    info[1] = F->n_vals;
    info[2] = F->analysis->levels;
    // Product launches a pass makes: one per tree level and direction.
    info[3] = F->launches_per_pass;
    return OB_OK;
}

int ob_chol_host_solve(int n, const int32_t* offsets, const int32_t* columns,
                       const double* values, const float* xyz, int leaf_size, int singular,
                       const double* rhs,
                       double* x, long long* info) {
    OB_REQUIRE(n >= 1 && offsets && columns && values && rhs && x, "ob_chol_host_solve: bad argument");
    std::vector<int> off(offsets, offsets + n + 1), col(columns, columns + offsets[n]);
    Analysis A;
    int st = analyse(n, std::move(off), std::move(col), xyz, leaf_size, &A);
    if (st) return st;
    HostFactor H;
    st = numeric(A, values, singular != 0, &H);
    if (st == OB_ERR_INDEFINITE) return fail(OB_ERR_INDEFINITE, "ob_chol_host_solve: not positive definite");
    if (st) return st;
    if (info) {
        info[0] = A.n;
        info[1] = (long long)A.nodes.size();
        info[2] = A.levels;
        info[3] = A.factor_entries;
    }
    // The device algorithm, run on the host: forward by levels' postorder (y1 = L11^-1 b1,
    // b2 += G b1), backward reversed (x1 = L11^-T y1 + G^T x2), G = -L21 L11^-1.
    std::vector<double> b(n), y(n, 0.0), xs(n, 0.0);
    for (int i = 0; i < n; ++i) b[i] = H.pinned[i] ? 0.0 : rhs[A.perm[i]];
    for (int s = 0; s < (int)A.nodes.size(); ++s) {
        const Node& nd = A.nodes[s];
        const int nc = nd.count, noff = (int)nd.off_rows.size();
        for (int i = 0; i < nc; ++i) {
            double acc = 0.0;
            for (int j = 0; j < nc; ++j) acc += H.inv[s][(size_t)i * nc + j] * b[nd.start + j];
            y[nd.start + i] = acc;
        }
        for (int r = 0; r < noff; ++r) {
            double acc = 0.0;
            for (int j = 0; j < nc; ++j) acc += H.off[s][(size_t)r * nc + j] * b[nd.start + j];
            b[nd.off_rows[r]] += acc;
        }
    }
    for (int s = (int)A.nodes.size() - 1; s >= 0; --s) {
        const Node& nd = A.nodes[s];
        const int nc = nd.count, noff = (int)nd.off_rows.size();
        for (int i = 0; i < nc; ++i) {
            double acc = 0.0;
            for (int j = 0; j < nc; ++j) acc += H.inv[s][(size_t)j * nc + i] * y[nd.start + j];
            for (int r = 0; r < noff; ++r) acc += H.off[s][(size_t)r * nc + i] * xs[nd.off_rows[r]];
            xs[nd.start + i] = acc;
        }
    }
    for (int i = 0; i < n; ++i) x[A.perm[i]] = xs[i];
    return OB_OK;
}

int ob_chol_values(void* factor, double* out, long long capacity, long long* count, ob_stream_t stream_) {
    OB_REQUIRE(factor && count, "ob_chol_values: bad argument");
    Factor* F = static_cast<Factor*>(factor);
    *count = F->n_vals;
    if (out == nullptr) return OB_OK;
    OB_REQUIRE(capacity >= F->n_vals, "ob_chol_values: %lld values need room, %lld given", F->n_vals, capacity);
    OB_CUDA(cudaMemcpyAsync(out, F->vals, sizeof(double) * (size_t)F->n_vals, cudaMemcpyDeviceToDevice,
                            as_stream(stream_)));
    return OB_OK;
}

int ob_chol_nbytes(void* factor, size_t* bytes) {
    OB_REQUIRE(factor && bytes, "ob_chol_nbytes: bad argument");
    *bytes = static_cast<Factor*>(factor)->bytes;
    return OB_OK;
}

int ob_chol_destroy(void* factor) {
    factor_release(static_cast<Factor*>(factor));
    return OB_OK;
}

}  // extern "C"
