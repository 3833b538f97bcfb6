// Host symbolic analysis: fill-reducing ordering, elimination tree, column
// counts and the (super/relaxed)nodal assembly tree, reproducing the reference
// bit for bit (mdgpu.cu:1745-1875, cs.cpp, etree.cpp).  Everything here runs
// once per sparsity pattern; the numeric work lives in the CUDA kernels.
#pragma once

#include <cstdint>
#include <vector>

namespace mdgpu {

// Compressed sparse column matrix, 32-bit indices (the reference's cs layout).
struct SparseCol {
    int nrows = 0, ncols = 0;
    std::vector<int> colptr;  // ncols + 1
    std::vector<int> rowidx;  // nnz
    std::vector<double> val;  // nnz or empty (pattern only)
    int nnz() const { return colptr.empty() ? 0 : colptr[ncols]; }
    bool has_values() const { return !val.empty(); }
};

SparseCol transpose(const SparseCol& A, bool values);
// Full symmetric matrix from its lower triangle (reference make_sym, mdgpu.cu:1630).
SparseCol symmetric_from_lower(const SparseCol& lower);
// Symmetric permutation of an upper-stored matrix, given the inverse
// permutation (cs_symperm, cs.cpp:1005).
SparseCol permute_upper(const SparseCol& upper, const std::vector<int>& inv_perm);

// Approximate-minimum-degree order of A + A' (cs_amd order 1, cs.cpp:645).
std::vector<int> amd_order(const SparseCol& upper);
// Elimination tree of a full symmetric pattern (cs_etree, cs.cpp:480).
std::vector<int> elimination_tree(const SparseCol& full);
// Postorder of a forest, children visited in ascending order (cs_post, cs.cpp:432).
std::vector<int> tree_postorder(const std::vector<int>& parent);
// Column counts of L (cs_counts with ata = 0, cs.cpp:338).
std::vector<int> column_counts(const SparseCol& full, const std::vector<int>& parent,
                               const std::vector<int>& post);

// Assembly tree: nodes in the order the multifrontal driver visits them
// (children before parents, the root last); node s eliminates the consecutive
// columns [first_col[s], first_col[s] + ncols[s]).
struct AssemblyTree {
    std::vector<int> first_col, ncols;
    std::vector<int> child_ptr, child;  // children of s, in visiting order
    int size() const { return (int)first_col.size(); }
};

enum class TreeKind { Nodal = 0, Super = 1, Relaxed = 2 };

// One column per node (GetETree, etree.cpp:12).
AssemblyTree nodal_tree(const std::vector<int>& parent, const std::vector<int>& post);
// Chains of columns with nested structure merged (GetSuperETree, etree.cpp:50).
AssemblyTree super_tree(const std::vector<int>& parent, const std::vector<int>& post,
                        const std::vector<int>& count);
// Greedy merge of children allowing up to max_zeros explicit zeros
// (GetRelaxedETree, etree.cpp:194).  Updates `count` (old numbering) and
// returns in `perm` the renumbering new -> old that makes every relaxed node
// a run of consecutive columns; the tree is in the new numbering.
AssemblyTree relaxed_tree(const std::vector<int>& parent, const std::vector<int>& post,
                          std::vector<int>& count, int max_zeros, std::vector<int>& perm);

// Output of the complete symbolic phase (mdgpu.cu:1745-1875).
struct Symbolic {
    int n = 0;
    std::vector<int> perm;            // new -> old, empty for natural order
    std::vector<int> parent, post;    // etree of the AMD-permuted matrix
    std::vector<int> count0, count;   // cs_counts output; counts used for L
    std::vector<int> relax_perm;      // GetRelaxedETree renumbering (relaxed only)
    SparseCol lower;                  // permuted lower triangle with values
    std::vector<int> lower_src;       // index of each lower entry in the user's array
    AssemblyTree tree;
    std::vector<int64_t> Lp;          // column pointers of L (cumsum of count)
};

// status 0 on success, -1 if the pattern is not a single tree (forest).
int analyze(int n, const int* Ap, const int* Ai, const double* Ax, bool use_amd,
            TreeKind kind, int relax_zeros, Symbolic& out);

}  // namespace mdgpu
