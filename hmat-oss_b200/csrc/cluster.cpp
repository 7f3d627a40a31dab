// Cluster tree (median bisection) and block tree of the B200 engine.  Host code; the
// arithmetic (bounding boxes, diameters, distances, axis choice) follows the reference
// operation by operation so that the permutation and the leaf list are identical.
#include <algorithm>
#include <cmath>

#include "host.h"

namespace hmatb200 {
namespace {

// AxisAlignedBoundingBox(const ClusterData&) (cluster_tree.cpp:212-230): first point, then
// std::min / std::max per coordinate.
void bounding_box(const ClusterTree& t, int offset, int size, double* bb) {
  const int* idx = t.perm.data() + offset;
  for (int d = 0; d < 3; ++d) bb[d] = bb[d + 3] = t.pts[3 * (size_t)idx[0] + d];
  for (int i = 1; i < size; ++i) {
    const double* p = &t.pts[3 * (size_t)idx[i]];
    for (int d = 0; d < 3; ++d) {
      bb[d] = std::min(bb[d], p[d]);
      bb[d + 3] = std::max(bb[d + 3], p[d]);
    }
  }
}

// largestDimension with avoidRatio 1.2 (clustering.cpp:135-152).
int largest_dimension(const double* bb, int to_avoid) {
  std::pair<double, int> e[3];
  for (int d = 0; d < 3; ++d) e[d] = std::make_pair(bb[d + 3] - bb[d], d);
  std::sort(e, e + 3);
  if (to_avoid < 0 || e[2].second != to_avoid || e[2].first > 1.2 * e[1].first) return e[2].second;
  return e[1].second;
}

struct Builder {
  ClusterTree& t;
  int max_leaf;
  void divide(int node, int axis) {
    const int offset = t.nodes[node].offset, size = t.nodes[node].size;
    if (size <= max_leaf) return;
    double bb[6];
    bounding_box(t, offset, size, bb);
    const int dim = largest_dimension(bb, axis);
    const double* pts = t.pts.data();
    // sortByDimension: stable sort on the coordinate (clustering.cpp:108-114)
    std::stable_sort(t.perm.begin() + offset, t.perm.begin() + offset + size,
                     [pts, dim](int a, int b) { return pts[3 * (size_t)a + dim] < pts[3 * (size_t)b + dim]; });
    const int middle = size / 2;
    int kids[2];
    int nk = 0;
    const int depth = t.nodes[node].depth + 1;
    if (middle > 0) {
      ClusterNode c;
      c.offset = offset;
      c.size = middle;
      c.depth = depth;
      t.nodes.push_back(c);
      kids[nk++] = (int)t.nodes.size() - 1;
    }
    {
      ClusterNode c;
      c.offset = offset + middle;
      c.size = size - middle;
      c.depth = depth;
      t.nodes.push_back(c);
      kids[nk++] = (int)t.nodes.size() - 1;
    }
    t.nodes[node].nchild = nk;
    for (int c = 0; c < nk; ++c) t.nodes[node].child[c] = kids[c];
    for (int c = 0; c < nk; ++c) divide(kids[c], dim);
  }
};

double diameter(const double* bb) {
  double r = 0.0;
  for (int i = 0; i < 3; ++i) {
    double d = bb[i] - bb[i + 3];
    r += d * d;
  }
  return std::sqrt(r);
}

double distance(const double* a, const double* b) {
  double r = 0.0;
  for (int i = 0; i < 3; ++i) {
    double d = std::max(0., a[i] - b[i + 3]);
    r += d * d;
    d = std::max(0., b[i] - a[i + 3]);
    r += d * d;
  }
  return std::sqrt(r);
}

struct BlockBuilder {
  const ClusterTree& R;
  const ClusterTree& C;
  const Admissibility& adm;
  BlockTree& out;

  void build(int rn, int cn) {
    const ClusterNode& r = R.nodes[rn];
    const ClusterNode& c = C.nodes[cn];
    out.nr_block_clusters++;
    if (r.size == 0 || c.size == 0) return;
    const double dmin = std::min(diameter(r.bb), diameter(c.bb));
    const bool low_rank = dmin > 0.0 && dmin <= adm.eta * distance(r.bb, c.bb);
    const bool rows_leaf = r.nchild == 0, cols_leaf = c.nchild == 0;
    const bool stop = r.size < 2 || c.size < 2;
    const bool force_rec = (size_t)r.size > adm.max_width || (size_t)c.size > adm.max_width;
    if ((rows_leaf && cols_leaf) || stop || (low_rank && !force_rec)) {
      const bool force_full = r.size < 2 || c.size < 2;
      LeafInfo L;
      L.row_node = rn;
      L.col_node = cn;
      L.row_off = r.offset;
      L.m = r.size;
      L.col_off = c.offset;
      L.n = c.size;
      L.type = (low_rank && !force_full) ? 1 : 0;
      out.leaves.push_back(L);
      return;
    }
    // splitRowsCols (admissibility.cpp:38-49)
    bool split_r, split_c;
    if (c.size < adm.ratio * r.size) {
      split_r = !rows_leaf;
      split_c = false;
    } else if (r.size < adm.ratio * c.size) {
      split_r = false;
      split_c = !cols_leaf;
    } else {
      split_r = !rows_leaf;
      split_c = !cols_leaf;
    }
    if (!split_r && !split_c) throw Error("block tree: cannot split a non-leaf block (check the ratio setting)");
    const int nr = split_r ? r.nchild : 1;
    const int nc = split_c ? c.nchild : 1;
    // child (i, j) is stored at i + j * nr and visited in storage order
    for (int j = 0; j < nc; ++j)
      for (int i = 0; i < nr; ++i) build(split_r ? r.child[i] : rn, split_c ? c.child[j] : cn);
  }
};

void collect_leaves(ClusterTree& t, int node) {
  const ClusterNode& nd = t.nodes[node];
  if (nd.nchild == 0) {
    t.leaf_nodes.push_back(node);
    return;
  }
  for (int c = 0; c < nd.nchild; ++c) collect_leaves(t, nd.child[c]);
}

}  // namespace

std::unique_ptr<ClusterTree> build_cluster_tree(const double* coord, int n, int max_leaf) {
  if (n <= 0) throw Error("cluster tree: no points");
  if (max_leaf < 1) throw Error("cluster tree: leaf size must be >= 1");
  std::unique_ptr<ClusterTree> t(new ClusterTree());
  t->n = n;
  t->pts.assign(coord, coord + 3 * (size_t)n);
  t->perm.resize(n);
  for (int i = 0; i < n; ++i) t->perm[i] = i;
  ClusterNode root;
  root.offset = 0;
  root.size = n;
  t->nodes.reserve(4 * (size_t)(n / std::max(1, max_leaf / 2) + 1));
  t->nodes.push_back(root);
  Builder b{*t, max_leaf};
  b.divide(0, -1);
  t->rev.resize(n);
  for (int i = 0; i < n; ++i) t->rev[t->perm[i]] = i;
  for (auto& nd : t->nodes)
    if (nd.size > 0) bounding_box(*t, nd.offset, nd.size, nd.bb);
  collect_leaves(*t, 0);
  return t;
}

BlockTree build_block_tree(const ClusterTree& rows, const ClusterTree& cols, const Admissibility& adm) {
  BlockTree bt;
  BlockBuilder b{rows, cols, adm, bt};
  b.build(0, 0);
  return bt;
}

}  // namespace hmatb200
