// Host-side structures of the B200 engine: cluster trees, admissibility, block tree.
// These stay on the CPU (they are O(N log N) integer / geometry work) and reproduce the
// reference's partition exactly; the device only ever sees the flattened leaf list.
#pragma once
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace hmatb200 {

struct ClusteringAlgo {
  int max_leaf = -1;  // -1: use the global maxLeafSize setting
  int divider = 2;
};

struct ClusterNode {
  int offset = 0, size = 0;
  int child[2] = {-1, -1};
  int nchild = 0;
  int depth = 0;
  double bb[6] = {0, 0, 0, 0, 0, 0};  // min xyz, max xyz
};

struct ClusterTree {
  int n = 0;
  std::vector<double> pts;  // client numbering, point-major xyz
  std::vector<int> perm;    // internal -> client
  std::vector<int> rev;     // client -> internal
  std::vector<ClusterNode> nodes;
  std::vector<int> leaf_nodes;  // tree leaves in cluster order
};

// Median bisection (clustering.cpp:108-152, 257-301, 488-565).
std::unique_ptr<ClusterTree> build_cluster_tree(const double* coord, int n, int max_leaf);

struct Admissibility {
  double eta = 2.0;
  double ratio = 0.0;
  size_t max_width = (size_t)-1;
};

struct LeafInfo {
  int row_node, col_node;
  int row_off, m, col_off, n;
  int type;  // 0 full, 1 rk
};

struct BlockTree {
  std::vector<LeafInfo> leaves;  // reference's depth-first (assembly) order
  int nr_block_clusters = 0;
};

// HMatrix construction (h_matrix.cpp:144-221) with the standard condition
// (admissibility.cpp:38-49, 95-117).
BlockTree build_block_tree(const ClusterTree& rows, const ClusterTree& cols, const Admissibility& adm);

struct Error : std::runtime_error {
  explicit Error(const std::string& s) : std::runtime_error(s) {}
};

}  // namespace hmatb200
