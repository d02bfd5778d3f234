// Host-side symbolic analysis for the multifrontal LDL^T: fill-reducing
// ordering, elimination tree, post-order, column counts, fundamental and
// relaxed supernodes, children lists and contribution-row lists.
//
// Every array produced here must equal the reference SparseLDL's arrays bit
// for bit (include/sparse_ldl.h:2204-2358 and include/block_amd.h:27-452),
// because the numeric factorization, the pivot order it implies and the
// inertia it reports are all defined on that structure.
#pragma once
#include <cstdint>
#include <vector>

namespace ab {

// Same numbering as the reference OrderingType (include/ordering_utils.h:21).
enum Ordering : int { ORDER_ND = 0, ORDER_AMD = 1, ORDER_MULTI_COLOR = 2,
                      ORDER_NATURAL = 3 };

struct SymbolicTree {
  int n = 0;
  int num_nodes = 0;
  bool permuted = false;
  std::vector<int> invperm;        // original var -> permuted index (size n)
  std::vector<int> node_ptr;       // num_nodes + 1
  std::vector<int> node_to_var;    // n, original numbering
  std::vector<int> children_ptr;   // num_nodes + 2; roots at the tail
  std::vector<int> children;       // num_nodes
  std::vector<int> contrib_ptr;    // num_nodes + 1
  std::vector<int> contrib_rows;   // original numbering, ascending permuted
  std::vector<int> node_parent;    // num_nodes (-1 for roots)
};

// Approximate-minimum-degree ordering on a pattern that already contains
// the diagonal and has sorted, unique rows.  `adj` is modified in place
// (it is the quotient-graph storage).  Returns 0 on success.
int amd_order(int n, std::vector<int>& rowp, std::vector<int>& adj,
              std::vector<int>& perm);

// Full fill-reducing ordering as the reference applies it inside SparseLDL:
// copy (adding or dropping the diagonal), sort/uniquify, then order.
void compute_ordering(int order, int n, const int* rowp, const int* cols,
                      std::vector<int>& perm, std::vector<int>& iperm);

// The full symbolic phase.  rowp/cols is the symmetric pattern (both
// triangles, rows need not be sorted).
void analyze(int order, int n, const int* rowp, const int* cols,
             SymbolicTree& out);

}  // namespace ab
