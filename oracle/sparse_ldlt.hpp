// ORACLE / TEST INFRASTRUCTURE ONLY.  Never linked into the product library.
//
// Sparse LDL^T factorisation standing in for Eigen::SimplicialLDLT, which the
// reference uses for scenes with fewer than 2000 local bodies
// (src/Solver/PrimalDual/PrimalDualForceSolver.cpp:385-394, src/Common/MatrixTypes.h:14).
// Eigen is absent here, so this is an own restatement of the published
// up-looking LDL^T algorithm (T. A. Davis, "Algorithm 849: A concise sparse
// Cholesky factorization package", ACM TOMS 31(4), 2005): elimination tree +
// row-pattern symbolic pass once per step (analyzePattern at it==0, :386-388)
// and a numeric pass every Newton iteration (factorize, :389).  Like
// SimplicialLDLT it reports failure only on an exactly zero pivot.
//
// The fill-reducing ordering is a greedy minimum-degree ordering of the 6x6
// block graph (Eigen uses AMD on the scalar graph); the ordering changes only
// round-off, never the solution.
#pragma once
#include <algorithm>
#include <cstdint>
#include <set>
#include <vector>

namespace pdc_oracle {

// Greedy minimum-degree ordering of an undirected graph given as adjacency
// lists (no self loops).  Ties are broken by the smallest node index so the
// ordering is deterministic.  Returns perm with perm[new] = old.
inline std::vector<int> min_degree_order(const std::vector<std::vector<int>>& adj) {
    const int n = (int)adj.size();
    std::vector<std::set<int>> g(n);
    for (int i = 0; i < n; ++i)
        for (int j : adj[i])
            if (j != i) { g[i].insert(j); g[j].insert(i); }
    std::set<std::pair<int, int>> pq;  // (degree, node)
    for (int i = 0; i < n; ++i) pq.insert({(int)g[i].size(), i});
    std::vector<char> done(n, 0);
    std::vector<int> perm;
    perm.reserve(n);
    while (!pq.empty()) {
        auto it = pq.begin();
        const int v = it->second;
        pq.erase(it);
        done[v] = 1;
        perm.push_back(v);
        std::vector<int> nb(g[v].begin(), g[v].end());
        for (int a : nb) {
            pq.erase({(int)g[a].size(), a});
            g[a].erase(v);
        }
        for (size_t x = 0; x < nb.size(); ++x)
            for (size_t y = x + 1; y < nb.size(); ++y) {
                g[nb[x]].insert(nb[y]);
                g[nb[y]].insert(nb[x]);
            }
        for (int a : nb) pq.insert({(int)g[a].size(), a});
        g[v].clear();
    }
    return perm;
}

// Scalar sparse symmetric matrix in compressed-column form, upper triangle
// only (row <= col), already permuted.
struct UpperCSC {
    int n = 0;
    std::vector<int> colptr, rowidx;
    std::vector<double> val;
};

class SparseLDLT {
   public:
    // Symbolic pass: elimination tree and column counts of L.
    void analyze(const UpperCSC& A) {
        n_ = A.n;
        parent_.assign(n_, -1);
        lnz_.assign(n_, 0);
        std::vector<int> flag(n_, -1);
        for (int k = 0; k < n_; ++k) {
            parent_[k] = -1;
            flag[k] = k;
            for (int p = A.colptr[k]; p < A.colptr[k + 1]; ++p) {
                int i = A.rowidx[p];
                if (i >= k) continue;
                for (; flag[i] != k; i = parent_[i]) {
                    if (parent_[i] == -1) parent_[i] = k;
                    lnz_[i]++;
                    flag[i] = k;
                }
            }
        }
        lp_.assign(n_ + 1, 0);
        for (int k = 0; k < n_; ++k) lp_[k + 1] = lp_[k] + lnz_[k];
        li_.assign(lp_[n_], 0);
        lx_.assign(lp_[n_], 0.0);
        d_.assign(n_, 0.0);
    }

    // Numeric pass.  Returns false on a zero pivot (Eigen: NumericalIssue).
    bool factorize(const UpperCSC& A) {
        std::vector<double> y(n_, 0.0);
        std::vector<int> pattern(n_), flag(n_, -1), cnt(n_, 0);
        for (int k = 0; k < n_; ++k) {
            y[k] = 0.0;
            int top = n_;
            flag[k] = k;
            cnt[k] = 0;
            for (int p = A.colptr[k]; p < A.colptr[k + 1]; ++p) {
                int i = A.rowidx[p];
                if (i > k) continue;
                y[i] += A.val[p];
                int len = 0;
                for (; flag[i] != k; i = parent_[i]) {
                    pattern[len++] = i;
                    flag[i] = k;
                }
                while (len > 0) pattern[--top] = pattern[--len];
            }
            d_[k] = y[k];
            y[k] = 0.0;
            for (; top < n_; ++top) {
                const int i = pattern[top];
                const double yi = y[i];
                y[i] = 0.0;
                const int p2 = lp_[i] + cnt[i];
                for (int p = lp_[i]; p < p2; ++p) y[li_[p]] -= lx_[p] * yi;
                const double lki = yi / d_[i];
                d_[k] -= lki * yi;
                li_[p2] = k;
                lx_[p2] = lki;
                cnt[i]++;
            }
            if (d_[k] == 0.0) return false;
        }
        return true;
    }

    // In-place solve of (L D L^T) x = b.
    void solve(std::vector<double>& x) const {
        for (int j = 0; j < n_; ++j)
            for (int p = lp_[j]; p < lp_[j + 1]; ++p) x[li_[p]] -= lx_[p] * x[j];
        for (int j = 0; j < n_; ++j) x[j] /= d_[j];
        for (int j = n_ - 1; j >= 0; --j)
            for (int p = lp_[j]; p < lp_[j + 1]; ++p) x[j] -= lx_[p] * x[li_[p]];
    }

    size_t nnz() const { return li_.size(); }

   private:
    int n_ = 0;
    std::vector<int> parent_, lnz_, lp_, li_;
    std::vector<double> lx_, d_;
};

}  // namespace pdc_oracle
