/* hmat_oracle.c -- CPU restatement of hmat-oss's leaf-level path (TEST INFRASTRUCTURE ONLY).
 *
 * Checker for the B200 engine: loaded only by tests/, the smoke check and the
 * benchmark's CPU-baseline leg.  See hmat_oracle.h for the reference functions each
 * part follows.  FP64 throughout; the complex path uses C99 double complex.
 */
#include "hmat_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int offset, size;
  int child[2];
  int nchild;
  double bb[6]; /* min x, y, z, max x, y, z */
} oracle_node;

typedef struct {
  int row_off, m, col_off, n;
  int type; /* 0 full, 1 rk */
  int rank; /* -1 for full leaves */
  void* data;
} oracle_leaf;

typedef struct {
  int leaf_size;
  int* perm; /* internal -> client */
  oracle_node* nodes;
  int nnodes, cap_nodes;
} oracle_tree;

struct oracle_hmat {
  int n, is_complex;
  double eta;
  double* pts; /* client numbering, point-major */
  oracle_tree rt, ct; /* row and column cluster trees (same points) */
  oracle_leaf* leaves;
  int nleaves, cap_leaves;
  int nr_block_clusters;
};

/* ------------------------------------------------------------------------------------ */
/* Cluster tree: median bisection (clustering.cpp:108-152,257-301,488-565).             */
/* ------------------------------------------------------------------------------------ */

static int new_node(oracle_tree* h, int offset, int size) {
  if (h->nnodes == h->cap_nodes) {
    h->cap_nodes = h->cap_nodes ? 2 * h->cap_nodes : 64;
    h->nodes = (oracle_node*)realloc(h->nodes, sizeof(oracle_node) * h->cap_nodes);
  }
  oracle_node* nd = &h->nodes[h->nnodes];
  nd->offset = offset;
  nd->size = size;
  nd->nchild = 0;
  nd->child[0] = nd->child[1] = -1;
  return h->nnodes++;
}

/* AxisAlignedBoundingBox(const ClusterData&) (cluster_tree.cpp:212-230) */
static void compute_bbox(const oracle_tree* h, const double* pts, int offset, int size, double* bb) {
  const int* idx = h->perm + offset;
  for (int d = 0; d < 3; ++d) bb[d] = bb[d + 3] = pts[3 * (size_t)idx[0] + d];
  for (int i = 1; i < size; ++i) {
    const double* p = pts + 3 * (size_t)idx[i];
    for (int d = 0; d < 3; ++d) {
      double v = p[d];
      bb[d] = v < bb[d] ? v : bb[d];           /* std::min(bb, v) */
      bb[d + 3] = bb[d + 3] < v ? v : bb[d + 3]; /* std::max(bb, v) */
    }
  }
}

/* largestDimension with avoidRatio 1.2 (clustering.cpp:135-152): sort (extent, dim) pairs
 * ascending, take the largest unless it is the axis to avoid and not 1.2x longer than the
 * second. */
static int largest_dimension(const double* bb, int toAvoid) {
  double e[3];
  int dm[3] = {0, 1, 2};
  for (int d = 0; d < 3; ++d) e[d] = bb[d + 3] - bb[d];
  for (int a = 1; a < 3; ++a) { /* lexicographic (extent, dim) order */
    double ev = e[a];
    int dv = dm[a];
    int b = a - 1;
    while (b >= 0 && (e[b] > ev || (e[b] == ev && dm[b] > dv))) {
      e[b + 1] = e[b];
      dm[b + 1] = dm[b];
      b--;
    }
    e[b + 1] = ev;
    dm[b + 1] = dv;
  }
  if (toAvoid < 0 || dm[2] != toAvoid || e[2] > 1.2 * e[1]) return dm[2];
  return dm[1];
}

/* Stable merge sort of idx[0..n) by pts[3*idx+dim] (the std::stable_sort of
 * sortByDimension, clustering.cpp:108-114). */
static void stable_sort_axis(int* idx, int n, const double* pts, int dim, int* tmp) {
  if (n < 2) return;
  int h = n / 2;
  stable_sort_axis(idx, h, pts, dim, tmp);
  stable_sort_axis(idx + h, n - h, pts, dim, tmp);
  int i = 0, j = h, o = 0;
  while (i < h && j < n) {
    /* take from the right only if strictly smaller: keeps equal keys in order */
    if (pts[3 * (size_t)idx[j] + dim] < pts[3 * (size_t)idx[i] + dim]) tmp[o++] = idx[j++];
    else tmp[o++] = idx[i++];
  }
  while (i < h) tmp[o++] = idx[i++];
  while (j < n) tmp[o++] = idx[j++];
  memcpy(idx, tmp, sizeof(int) * n);
}

static void divide_recursive(oracle_tree* h, const double* pts, int node, int currentAxis, int* tmp) {
  int offset = h->nodes[node].offset, size = h->nodes[node].size;
  if (size <= h->leaf_size) return;
  double bb[6];
  compute_bbox(h, pts, offset, size, bb);
  int dim = largest_dimension(bb, currentAxis);
  stable_sort_axis(h->perm + offset, size, pts, dim, tmp);
  int middle = size / 2; /* size * i / divider with divider 2 */
  int c0 = -1, c1;
  if (middle > 0) c0 = new_node(h, offset, middle);
  c1 = new_node(h, offset + middle, size - middle);
  int k = 0;
  if (c0 >= 0) h->nodes[node].child[k++] = c0;
  h->nodes[node].child[k++] = c1;
  h->nodes[node].nchild = k;
  for (int c = 0; c < k; ++c) divide_recursive(h, pts, h->nodes[node].child[c], dim, tmp);
}

/* ------------------------------------------------------------------------------------ */
/* Block tree (h_matrix.cpp:144-221) with the Hackbusch condition (admissibility.cpp). */
/* ------------------------------------------------------------------------------------ */

static double bb_diameter(const double* bb) {
  double r = 0.0;
  for (int i = 0; i < 3; ++i) {
    double d = bb[i] - bb[i + 3];
    r += d * d;
  }
  return sqrt(r);
}

static double bb_distance(const double* a, const double* b) {
  double r = 0.0;
  for (int i = 0; i < 3; ++i) {
    double d = a[i] - b[i + 3];
    d = d > 0.0 ? d : 0.0;
    r += d * d;
    d = b[i] - a[i + 3];
    d = d > 0.0 ? d : 0.0;
    r += d * d;
  }
  return sqrt(r);
}

static void add_leaf(oracle_hmat* h, int rn, int cn, int type) {
  if (h->nleaves == h->cap_leaves) {
    h->cap_leaves = h->cap_leaves ? 2 * h->cap_leaves : 256;
    h->leaves = (oracle_leaf*)realloc(h->leaves, sizeof(oracle_leaf) * h->cap_leaves);
  }
  oracle_leaf* L = &h->leaves[h->nleaves++];
  L->row_off = h->rt.nodes[rn].offset;
  L->m = h->rt.nodes[rn].size;
  L->col_off = h->ct.nodes[cn].offset;
  L->n = h->ct.nodes[cn].size;
  L->type = type;
  L->rank = type == 0 ? -1 : 0;
  L->data = NULL;
}

static void build_block(oracle_hmat* h, int rn, int cn) {
  const oracle_node* R = &h->rt.nodes[rn];
  const oracle_node* C = &h->ct.nodes[cn];
  h->nr_block_clusters++;
  if (R->size == 0 || C->size == 0) return; /* isVoid */
  double dr = bb_diameter(R->bb), dc = bb_diameter(C->bb);
  double mind = dr < dc ? dr : dc;
  int lowRank = mind > 0.0 && mind <= h->eta * bb_distance(R->bb, C->bb);
  int rowsLeaf = R->nchild == 0, colsLeaf = C->nchild == 0;
  int stop = R->size < 2 || C->size < 2;
  if ((rowsLeaf && colsLeaf) || stop || lowRank) {
    int forceFull = R->size < 2 || C->size < 2;
    add_leaf(h, rn, cn, (lowRank && !forceFull) ? 1 : 0);
    return;
  }
  /* ratio 0: split every side that is not a leaf; child (i, j) stored at i + j * nrows,
   * visited in storage order as HMatrix::assemble does */
  int nr = rowsLeaf ? 1 : R->nchild;
  int nc = colsLeaf ? 1 : C->nchild;
  for (int j = 0; j < nc; ++j)
    for (int i = 0; i < nr; ++i) {
      int rc = rowsLeaf ? rn : R->child[i];
      int cc = colsLeaf ? cn : C->child[j];
      build_block(h, rc, cc);
    }
}

static void build_tree(oracle_tree* t, const double* pts, int n, int leaf_size) {
  t->leaf_size = leaf_size;
  t->perm = (int*)malloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; ++i) t->perm[i] = i;
  int* tmp = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int root = new_node(t, 0, n);
  divide_recursive(t, pts, root, -1, tmp);
  free(tmp);
  for (int i = 0; i < t->nnodes; ++i)
    if (t->nodes[i].size > 0) compute_bbox(t, pts, t->nodes[i].offset, t->nodes[i].size, t->nodes[i].bb);
}

oracle_hmat* oracle_create2(const double* pts, int n, int leaf_rows, int leaf_cols, double eta) {
  oracle_hmat* h = (oracle_hmat*)calloc(1, sizeof(oracle_hmat));
  h->n = n;
  h->eta = eta;
  h->pts = (double*)malloc(sizeof(double) * 3 * (size_t)n);
  memcpy(h->pts, pts, sizeof(double) * 3 * (size_t)n);
  build_tree(&h->rt, h->pts, n, leaf_rows);
  build_tree(&h->ct, h->pts, n, leaf_cols);
  build_block(h, 0, 0);
  return h;
}

oracle_hmat* oracle_create(const double* pts, int n, int leaf_size, double eta) {
  return oracle_create2(pts, n, leaf_size, leaf_size, eta);
}

void oracle_destroy(oracle_hmat* h) {
  if (!h) return;
  for (int i = 0; i < h->nleaves; ++i) free(h->leaves[i].data);
  free(h->leaves);
  free(h->rt.nodes);
  free(h->rt.perm);
  free(h->ct.nodes);
  free(h->ct.perm);
  free(h->pts);
  free(h);
}

void oracle_perm(const oracle_hmat* h, int* out) { memcpy(out, h->rt.perm, sizeof(int) * (size_t)h->n); }
void oracle_perm_cols(const oracle_hmat* h, int* out) { memcpy(out, h->ct.perm, sizeof(int) * (size_t)h->n); }

int oracle_num_leaves(const oracle_hmat* h) { return h->nleaves; }

void oracle_leaves(const oracle_hmat* h, int* out) {
  for (int i = 0; i < h->nleaves; ++i) {
    const oracle_leaf* L = &h->leaves[i];
    out[6 * i + 0] = L->row_off;
    out[6 * i + 1] = L->m;
    out[6 * i + 2] = L->col_off;
    out[6 * i + 3] = L->n;
    out[6 * i + 4] = L->type;
    out[6 * i + 5] = L->rank;
  }
}

int oracle_num_nodes(const oracle_hmat* h) { return h->rt.nnodes; }

void oracle_nodes(const oracle_hmat* h, int* out) {
  for (int i = 0; i < h->rt.nnodes; ++i) {
    out[4 * i + 0] = h->rt.nodes[i].offset;
    out[4 * i + 1] = h->rt.nodes[i].size;
    out[4 * i + 2] = h->rt.nodes[i].child[0];
    out[4 * i + 3] = h->rt.nodes[i].child[1];
  }
}

/* HMatrix::info (h_matrix.cpp:464-502) */
void oracle_info(const oracle_hmat* h, long long* out) {
  long long full_count = 0, rk_count = 0, full_size = 0, rk_size = 0, compressed = 0, uncompressed = 0;
  long long dim_r = 0, dim_c = 0, mem_r = 0, mem_c = 0, mem_k = 0;
  for (int i = 0; i < h->nleaves; ++i) {
    const oracle_leaf* L = &h->leaves[i];
    long long s = (long long)L->m * L->n;
    uncompressed += s;
    if (L->type == 1) {
      long long mem = (long long)L->rank * (L->m + L->n);
      compressed += mem;
      if (L->m + L->n > dim_r + dim_c) { dim_c = L->n; dim_r = L->m; }
      long long old = (mem_c + mem_r) * mem_k;
      if (mem > old) { mem_c = L->n; mem_r = L->m; mem_k = L->rank; }
      rk_count++;
      rk_size += s;
    } else {
      compressed += s;
      full_count++;
      full_size += s;
    }
  }
  out[0] = full_count; out[1] = rk_count; out[2] = full_size; out[3] = rk_size;
  out[4] = compressed; out[5] = uncompressed; out[6] = h->nr_block_clusters;
  out[7] = dim_r; out[8] = dim_c; out[9] = mem_r; out[10] = mem_c; out[11] = mem_k;
}

/* ------------------------------------------------------------------------------------ */
/* Kernels.                                                                              */
/* ------------------------------------------------------------------------------------ */

static const double kFourPi = 4.0 * M_PI;

static double point_dist(const double* a, const double* b) {
  double dx = a[0] - b[0];
  double dy = a[1] - b[1];
  double dz = a[2] - b[2];
  double s = dx * dx;
  s = s + dy * dy;
  s = s + dz * dz;
  return sqrt(s);
}

static double real_eval(const oracle_hmat* h, const oracle_kernel* k, int row, int col) {
  double r = point_dist(h->pts + 3 * (size_t)row, h->pts + 3 * (size_t)col);
  if (k->kind == 0) return 1.0 / (kFourPi * (r + k->delta));
  double v = exp(-r / k->ell);
  if (row == col) v += k->nugget;
  return v;
}

static double complex complex_eval(const oracle_hmat* h, const oracle_kernel* k, int row, int col) {
  double r = point_dist(h->pts + 3 * (size_t)row, h->pts + 3 * (size_t)col);
  double s = 1.0 / (kFourPi * (r + k->delta));
  double kr = k->wavenumber * r;
  return CMPLX(cos(kr) * s, sin(kr) * s);
}

/* Stratum `stratum` of a multi-strata kernel, or the sum of its strata in order for -1
 * (the callback convention of hmat.h:552-583). */
static double real_eval_s(const oracle_hmat* h, const oracle_kernel* k, int row, int col, int stratum) {
  if (k->nstrata < 1) return real_eval(h, k, row, col);
  double r = point_dist(h->pts + 3 * (size_t)row, h->pts + 3 * (size_t)col);
  double sum = 0.0;
  for (int q = 0; q < k->nstrata; ++q) {
    if (stratum >= 0 && q != stratum) continue;
    double w = k->sweight[q], a = k->sparam[q];
    double v = k->kind == 0 ? w * (1.0 / (kFourPi * (r + a))) : w * exp(-r / a);
    if (stratum >= 0) return v;
    sum = sum + v;
  }
  return sum;
}

static double complex complex_eval_s(const oracle_hmat* h, const oracle_kernel* k, int row, int col, int stratum) {
  if (k->nstrata < 1) return complex_eval(h, k, row, col);
  double r = point_dist(h->pts + 3 * (size_t)row, h->pts + 3 * (size_t)col);
  double sc = 1.0 / (kFourPi * (r + k->delta));
  double re = 0.0, im = 0.0;
  for (int q = 0; q < k->nstrata; ++q) {
    if (stratum >= 0 && q != stratum) continue;
    double w = k->sweight[q], kr = k->sparam[q] * r;
    double vr = w * (cos(kr) * sc), vi = w * (sin(kr) * sc);
    if (stratum >= 0) return CMPLX(vr, vi);
    re = re + vr;
    im = im + vi;
  }
  return CMPLX(re, im);
}

void oracle_kernel_eval(const oracle_hmat* h, const oracle_kernel* k, int row, int col, double* out) {
  if (k->kind == 2) {
    double complex v = complex_eval_s(h, k, row, col, -1);
    out[0] = creal(v);
    out[1] = cimag(v);
  } else {
    out[0] = real_eval_s(h, k, row, col, -1);
  }
}

static double complex complex_recip(double complex z) {
  double d = creal(z) * creal(z) + cimag(z) * cimag(z);
  return CMPLX(creal(z) / d, -cimag(z) / d);
}

/* ---- instantiate the leaf algorithms for double ---- */
#define SC double
#define FN(x) x##_r
#define ABS2(x) ((x) * (x))
#define CONJ(x) (x)
#define REALP(x) (x)
#define IAMAX_KEY(x) fabs(x)
#define RECIP(x) (1.0 / (x))
#define SC_EVAL(h, k, r, c, s) real_eval_s(h, k, r, c, s)
#include "oracle_leaf.inc"
#undef SC
#undef FN
#undef ABS2
#undef CONJ
#undef REALP
#undef IAMAX_KEY
#undef RECIP
#undef SC_EVAL

/* ---- and for double complex ---- */
#define SC double complex
#define FN(x) x##_c
#define ABS2(x) (creal(x) * creal(x) + cimag(x) * cimag(x))
#define CONJ(x) conj(x)
#define REALP(x) creal(x)
#define IAMAX_KEY(x) (fabs(creal(x)) + fabs(cimag(x)))
#define RECIP(x) complex_recip(x)
#define SC_EVAL(h, k, r, c, s) complex_eval_s(h, k, r, c, s)
#include "oracle_leaf.inc"
#undef SC
#undef FN
#undef ABS2
#undef CONJ
#undef REALP
#undef IAMAX_KEY
#undef RECIP
#undef SC_EVAL

int oracle_assemble2(oracle_hmat* h, const oracle_kernel* k, double epsilon, int is_complex, int min_leaf) {
  if (is_complex != (k->kind == 2)) return 1;
  h->is_complex = is_complex;
  for (int i = 0; i < h->nleaves; ++i) {
    if (is_complex) assemble_leaf_c(h, k, &h->leaves[i], epsilon, min_leaf);
    else assemble_leaf_r(h, k, &h->leaves[i], epsilon, min_leaf);
  }
  return 0;
}

int oracle_assemble(oracle_hmat* h, const oracle_kernel* k, double epsilon, int is_complex) {
  return oracle_assemble2(h, k, epsilon, is_complex, 0);
}

int oracle_retruncate(oracle_hmat* h, double epsilon) {
  for (int i = 0; i < h->nleaves; ++i) {
    if (h->is_complex) retruncate_leaf_c(&h->leaves[i], epsilon);
    else retruncate_leaf_r(&h->leaves[i], epsilon);
  }
  return 0;
}

long long oracle_leaf_payload_size(const oracle_hmat* h, int i) {
  const oracle_leaf* L = &h->leaves[i];
  if (!L->data) return 0;
  return L->type == 0 ? (long long)L->m * L->n : (long long)L->rank * (L->m + L->n);
}

void oracle_leaf_payload(const oracle_hmat* h, int i, double* out) {
  long long s = oracle_leaf_payload_size(h, i);
  if (s) memcpy(out, h->leaves[i].data, (size_t)s * (h->is_complex ? 16 : 8));
}

/* gemv in client numbering (c_wrapping.hpp:233-252): permute into cluster order, sum
 * the leaves, permute back. */
int oracle_gemv(const oracle_hmat* h, char trans, int nrhs, const double* x, double* y) {
  const int N = h->n;
  const size_t w = h->is_complex ? 2 : 1;
  const int* pin = trans == 'N' ? h->ct.perm : h->rt.perm;
  const int* pout = trans == 'N' ? h->rt.perm : h->ct.perm;
  double* xi = (double*)malloc(sizeof(double) * w * (size_t)N * nrhs);
  double* yi = (double*)calloc(w * (size_t)N * nrhs, sizeof(double));
  for (int r = 0; r < nrhs; ++r)
    for (int i = 0; i < N; ++i)
      for (size_t c = 0; c < w; ++c)
        xi[w * ((size_t)r * N + i) + c] = x[w * ((size_t)r * N + pin[i]) + c];
  for (int l = 0; l < h->nleaves; ++l) {
    if (h->is_complex)
      gemv_leaf_c(&h->leaves[l], trans, nrhs, (const double complex*)xi, (double complex*)yi, N);
    else
      gemv_leaf_r(&h->leaves[l], trans == 'C' ? 'T' : trans, nrhs, xi, yi, N);
  }
  for (int r = 0; r < nrhs; ++r)
    for (int i = 0; i < N; ++i)
      for (size_t c = 0; c < w; ++c)
        y[w * ((size_t)r * N + pout[i]) + c] = yi[w * ((size_t)r * N + i) + c];
  free(xi);
  free(yi);
  return 0;
}
