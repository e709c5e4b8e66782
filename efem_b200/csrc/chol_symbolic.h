// Host-side symbolic analysis for the approximate-Jacobian Cholesky factor.
//
// The reference factors K~ = L (x) I3 (3 DOF per node) with Eigen's
// SimplicialLLT and AMD ordering (src/simulation/nlsolver/LBFGS.h:65-81).
// Here the scalar node matrix L is factored instead -- the same H0 up to
// rounding, with 27x fewer factor flops -- after a geometric nested-dissection
// ordering that keeps the elimination tree shallow and wide for the GPU.
#pragma once
#include <vector>

namespace efem {

struct Symbolic {
    int n = 0;                         // free nodes
    std::vector<int> perm, iperm;      // new -> old, old -> new
    int ns = 0;                        // supernodes (fronts)
    std::vector<int> first, ncol, nrow;
    std::vector<long long> front_off;  // r x r column-major front per supernode
    std::vector<long long> rows_off;
    std::vector<int> rows;             // per front: its columns, then its below rows (new numbering, sorted)
    std::vector<int> parent;           // supernode parent, -1 for a root
    std::vector<int> child_ptr, child_list;
    std::vector<long long> relind_off;
    std::vector<int> relind;           // below rows of a front -> positions in the parent's rows
    std::vector<long long> dinv_off;   // c x c inverse of each diagonal block
    std::vector<long long> upd_off;    // (r - c) x 3 forward-solve update vector
    std::vector<long long> lt_off;     // row-major copy of each front's L_RJ ((r - c) x c)
    // for every front row (indexed rows_off[s] + t): the update-vector entries
    // of the children that land on it, in child order (CSR over rows)
    std::vector<int> contrib_ptr;
    std::vector<int> contrib_idx;      // index of a node-triple in the update array (upd_off/3 + j)
    std::vector<int> below_front;      // for each such index, the front whose update array holds it
    std::vector<int> level_ptr, level_list;  // fronts grouped by level, leaves first
    long long front_size = 0, dinv_size = 0, upd_size = 0, lt_size = 0, nnz_L = 0;
    double flops = 0;
    // original entries: front position of each lower-triangle entry of the CSR
    std::vector<long long> a_pos;
    std::vector<long long> a_src;      // index into the CSR value array
};

// Build the symbolic factor of the n x n symmetric matrix with CSR pattern
// (rowptr, col) (both triangles); coords (n x 3) drive the dissection.
void symbolic_analysis(int n, const std::vector<int>& rowptr, const std::vector<int>& col, const double* coords,
    Symbolic& S);

}  // namespace efem
