// C ABI of the B200 engine: the hmat-oss C entry points on the leaf-level path (same
// names, argument meaning and 0 / non-zero return convention as c_default_interface.cpp
// and c_wrapping.hpp) plus the hmat_b200_* extensions declared in include/hmat_b200.h.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "engine.h"
#include "hmat_b200.h"
#include "host.h"

using namespace hmatb200;

struct hmat_clustering_algorithm {
  ClusteringAlgo a;
};
struct hmat_cluster_tree_struct {
  std::unique_ptr<ClusterTree> t;
};
struct hmat_admissibility_condition {
  Admissibility a;
};
struct hmat_compression_algorithm_struct {
  hmat_compress_t method;
  double eps;
};
struct hmat_matrix_struct {
  int vt = 1;
  const hmat_cluster_tree_t* rows_h = nullptr;
  const hmat_cluster_tree_t* cols_h = nullptr;
  bool own_rows = false, own_cols = false;
  BlockTree bt;
  double low_rank_eps = 1e-4;  // LocalSettings default (h_matrix.cpp:151)
  std::unique_ptr<EngineBase> engine;
  // A batch (hmat_b200_batch_create): the first row and the first leaf of each member matrix
  // in the block-diagonal combination (count + 1 entries each); empty for a plain matrix.
  std::vector<int> batch_rows, batch_leaves;
};

namespace {

const unsigned kAssemblyMagic = 0xB200A55Eu;
struct AssemblyObj {
  unsigned magic = kAssemblyMagic;
  AssemblyDesc d;
};

thread_local std::string g_last_error;

// Global settings with the reference's defaults (hmat_cpp_interface.hpp:88-95).
hmat_settings_t g_settings = {100, 1e-4, 200, 0, 0, 0, 0, 0, 0, 0, 0.0};

// The device side of a matrix is created on first use, so that the host-only parts
// (clustering, block tree, leaf table) work without a GPU.
EngineBase& engine_of(hmat_matrix_t* m) {
  if (!m->engine) m->engine = make_engine(m->vt, m->rows_h->t.get(), m->cols_h->t.get(), &m->bt);
  return *m->engine;
}

int leaf_rank(const hmat_matrix_t* m, size_t i) {
  if (m->engine) return m->engine->ranks[i];
  return m->bt.leaves[i].type == 1 ? 0 : -1;
}

int fail(const char* where, const std::string& msg) {
  g_last_error = std::string(where) + ": " + msg;
  fprintf(stderr, "%s\n", g_last_error.c_str());
  return 1;
}

#define HB_TRY(where, ...)            \
  try {                               \
    __VA_ARGS__;                      \
  } catch (const std::exception& e) { \
    return fail(where, e.what());     \
  }


// ---- table entries on the path ----

hmat_matrix_t* create_empty(const hmat_cluster_tree_t* rows, const hmat_cluster_tree_t* cols, int lower_sym,
                            hmat_admissibility_t* cond, int vt) {
  try {
    if (!rows || !cols || !cond) throw Error("null argument");
    if (lower_sym) throw Error("lower-symmetric storage is not supported by the B200 engine");
    std::unique_ptr<hmat_matrix_t> m(new hmat_matrix_t());
    m->vt = vt;
    m->rows_h = rows;
    m->cols_h = cols;
    m->bt = build_block_tree(*rows->t, *cols->t, cond->a);
    return m.release();
  } catch (const std::exception& e) {
    fail("create_empty_hmatrix_admissibility", e.what());
    return nullptr;
  }
}
template <int VT>
hmat_matrix_t* create_empty_t(const hmat_cluster_tree_t* rows, const hmat_cluster_tree_t* cols, int lower_sym,
                              hmat_admissibility_t* cond) {
  return create_empty(rows, cols, lower_sym, cond, VT);
}

void own_cluster_trees(hmat_matrix_t* m, int owns_row, int owns_col) {
  if (!m) return;
  m->own_rows = owns_row != 0;
  m->own_cols = owns_col != 0;
}

void set_low_rank_epsilon(hmat_matrix_t* m, double eps) {
  if (m) m->low_rank_eps = eps;
}

int assemble_generic(hmat_matrix_t* m, hmat_assemble_context_t* ctx) {
  HB_TRY("assemble_generic", {
    if (!m || !ctx) throw Error("null argument");
    if (ctx->lower_symmetric) throw Error("lower-symmetric assembly is not supported by the B200 engine");
    if (!ctx->compression) throw Error("No compression algorithm defined in hmat_assemble_context_t");
    if (ctx->factorization != hmat_factorization_none)
      throw Error("factorization is outside the B200 engine's path");
    if (ctx->simple_compute || ctx->block_compute || ctx->advanced_compute)
      throw Error("host interaction callbacks cannot run on the device; pass hmat_b200_create_assembly() in "
                  "the 'assembly' field (hmat_b200_create_assembly_strata() for a multi-strata kernel)");
    const AssemblyObj* a = (const AssemblyObj*)ctx->assembly;
    if (!a || a->magic != kAssemblyMagic) throw Error("'assembly' is not a descriptor from hmat_b200_create_assembly");
    int method;
    switch (ctx->compression->method) {
      case hmat_compress_aca_plus: method = 0; break;
      case hmat_compress_aca_partial: method = 1; break;
      default: throw Error("only ACA+ and partial-ACA compression are implemented by the B200 engine");
    }
    const int svd_below = g_settings.compressionMinLeafSize;
    engine_of(m).assemble(a->d, method, ctx->compression->eps, m->low_rank_eps, svd_below);
  });
  return 0;
}

int destroy(hmat_matrix_t* m) {
  if (!m) return 0;
  const hmat_cluster_tree_t* r = m->own_rows ? m->rows_h : nullptr;
  const hmat_cluster_tree_t* c = m->own_cols ? m->cols_h : nullptr;
  delete m;
  if (r) hmat_delete_cluster_tree(r);
  if (c && c != r) hmat_delete_cluster_tree(c);
  return 0;
}

int gemv(char trans, void* alpha, hmat_matrix_t* m, void* x, void* beta, void* y, int nrhs) {
  HB_TRY("gemv", {
    if (!m || !alpha || !beta || (nrhs > 0 && (!x || !y))) throw Error("null argument");
    engine_of(m).gemv_host(trans, alpha, x, beta, y, nrhs);
  });
  return 0;
}

template <int VT>
int gemv_t(char trans, void* alpha, hmat_matrix_t* m, void* x, void* beta, void* y, int nrhs) {
  if (m && m->vt != VT) return fail("gemv", "matrix value type does not match this interface");
  return gemv(trans, alpha, m, x, beta, y, nrhs);
}

template <typename T>
void permute(T* v, const std::vector<int>& idx, int rows, int cols, int axis, bool restore) {
  const int n = axis == 0 ? rows : cols;
  std::vector<T> tmp(n);
  const int outer = axis == 0 ? cols : rows;
  for (int o = 0; o < outer; ++o) {
    for (int i = 0; i < n; ++i) {
      size_t a = axis == 0 ? (size_t)o * rows + i : (size_t)i * rows + o;
      size_t b = axis == 0 ? (size_t)o * rows + idx[i] : (size_t)idx[i] * rows + o;
      if (restore) tmp[idx[i]] = v[a];
      else tmp[i] = v[b];
    }
    for (int i = 0; i < n; ++i) v[axis == 0 ? (size_t)o * rows + i : (size_t)i * rows + o] = tmp[i];
  }
}

// reorderVector / restoreVectorOrder over a rows x cols column-major array
// (h_matrix.cpp:75-141, c_wrapping.hpp:455-500).
template <typename T>
int reorder_impl(void* vec, const hmat_cluster_tree_t* rct, int rows, const hmat_cluster_tree_t* cct, int cols,
                 bool restore) {
  HB_TRY(restore ? "vector_restore" : "vector_reorder", {
    if (!rct && rows == 0) throw Error("either row cluster tree or rows must be non null");
    if (!cct && cols == 0) throw Error("either col cluster tree or cols must be non null");
    const int nr = rct ? rct->t->n : rows, nc = cct ? cct->t->n : cols;
    if (rct) permute((T*)vec, rct->t->perm, nr, nc, 0, restore);
    if (cct) permute((T*)vec, cct->t->perm, nr, nc, 1, restore);
  });
  return 0;
}
template <typename T>
int vector_reorder_t(void* v, const hmat_cluster_tree_t* r, int rows, const hmat_cluster_tree_t* c, int cols) {
  return reorder_impl<T>(v, r, rows, c, cols, false);
}
template <typename T>
int vector_restore_t(void* v, const hmat_cluster_tree_t* r, int rows, const hmat_cluster_tree_t* c, int cols) {
  return reorder_impl<T>(v, r, rows, c, cols, true);
}

// HMatrix::info (h_matrix.cpp:464-502) over the flattened leaves.
int get_info(hmat_matrix_t* m, hmat_info_t* info) {
  HB_TRY("get_info", {
    if (!m || !info) throw Error("null argument");
    memset(info, 0, sizeof(*info));
    info->nr_block_clusters = m->bt.nr_block_clusters;
    const auto& L = m->bt.leaves;
    for (size_t i = 0; i < L.size(); ++i) {
      const size_t r = L[i].m, c = L[i].n;
      if (!r || !c) continue;
      const size_t s = r * c;
      info->uncompressed_size += s;
      if (L[i].type == 1) {
        const int k = leaf_rank(m, i);
        const size_t mem = (size_t)k * (r + c);
        info->compressed_size += mem;
        if ((int)(r + c) > info->largest_rk_dim_cols + info->largest_rk_dim_rows) {
          info->largest_rk_dim_cols = (int)c;
          info->largest_rk_dim_rows = (int)r;
        }
        const size_t old =
            ((size_t)info->largest_rk_mem_cols + info->largest_rk_mem_rows) * info->largest_rk_mem_rank;
        if (mem > old) {
          info->largest_rk_mem_cols = (int)c;
          info->largest_rk_mem_rows = (int)r;
          info->largest_rk_mem_rank = k;
        }
        info->rk_count++;
        info->rk_size += s;
      } else {
        info->compressed_size += s;
        info->full_count++;
        info->full_size += s;
      }
    }
  });
  return 0;
}

int get_cluster_trees(hmat_matrix_t* m, const hmat_cluster_tree_t** rows, const hmat_cluster_tree_t** cols) {
  if (!m) return fail("get_cluster_trees", "null matrix");
  if (rows) *rows = m->rows_h;
  if (cols) *cols = m->cols_h;
  return 0;
}

int init_fn(void) { return 0; }
int finalize_fn(void) { return 0; }

// ---- slots outside the path: explicit failures ----
int unsupported(const char* name) {
  return fail(name, "not supported by the B200 engine (outside the leaf-level assembly / gemv path)");
}
hmat_matrix_t* u_copy(hmat_matrix_t*) {
  unsupported("copy");
  return nullptr;
}
hmat_matrix_t* u_copy_struct(hmat_matrix_t*) {
  unsupported("copy_struct");
  return nullptr;
}
double u_norm(hmat_matrix_t*) {
  unsupported("norm");
  return -1.0;
}
int u_logdet(hmat_matrix_t*, double*) { return unsupported("logdet"); }
int u_inverse(hmat_matrix_t*) { return unsupported("inverse"); }
int u_factorize(hmat_matrix_t*, hmat_factorization_context_t*) { return unsupported("factorize_generic"); }
hmat_matrix_t* u_get_child(hmat_matrix_t*, int, int) {
  unsupported("get_child");
  return nullptr;
}
int u_destroy_child(hmat_matrix_t*) { return unsupported("destroy_child"); }
int u_solve_generic(hmat_matrix_t*, const struct hmat_solve_context_t*) { return unsupported("solve_generic"); }
int u_solve_mat(hmat_matrix_t*, hmat_matrix_t*) { return unsupported("solve_mat"); }
int u_solve_systems(hmat_matrix_t*, void*, int) { return unsupported("solve_systems"); }
int u_solve_dense(hmat_matrix_t*, void*, int) { return unsupported("solve_dense"); }
int u_transpose(hmat_matrix_t*) { return unsupported("transpose"); }
int u_scale(void*, hmat_matrix_t*) { return unsupported("scale"); }
// HMatInterface::truncate (hmat_cpp_interface.cpp:225-229 -> HMatrix::truncate,
// h_matrix.cpp:2107-2123): every Rk leaf re-truncated at the matrix's low-rank epsilon.
int c_truncate(hmat_matrix_t* m) {
  HB_TRY("truncate", {
    if (!m) throw Error("null argument");
    EngineBase* e = m->engine.get();
    if (!e || !e->assembled) throw Error("truncate needs an assembled matrix");
    e->retruncate(m->low_rank_eps);
  });
  return 0;
}
int u_gemm(char, char, const void*, hmat_matrix_t*, hmat_matrix_t*, const void*, hmat_matrix_t*) {
  return unsupported("gemm");
}
int u_axpy(void*, hmat_matrix_t*, hmat_matrix_t*) { return unsupported("axpy"); }
int u_trsm(char, char, char, char, int, int, void*, hmat_matrix_t*, int, void*) { return unsupported("trsm"); }

int u_full_gemm(char, char, int, int, void*, void*, void*, hmat_matrix_t*, void*) { return unsupported("full_gemm"); }
// ---- products and extraction in the H-matrix's internal (cluster) numbering ----
// Host scalar type of each value type (layout-identical to the device types).
template <int VT> struct HostScalar;
template <> struct HostScalar<0> { typedef float type; };
template <> struct HostScalar<1> { typedef double type; };
template <> struct HostScalar<2> { typedef std::complex<float> type; };
template <> struct HostScalar<3> { typedef std::complex<double> type; };
inline float conj_s(float v) { return v; }
inline double conj_s(double v) { return v; }
template <typename R>
std::complex<R> conj_s(std::complex<R> v) { return std::conj(v); }

bool flag_trans(char t) { return t == 'T' || t == 'C'; }
bool flag_conj(char t) { return t == 'C' || t == 'J'; }
// switch_flag_trans / switch_flag_conj (c_wrapping.hpp:280-298)
char switch_trans(char t) {
  switch (t) {
    case 'N': return 'T';
    case 'T': return 'N';
    case 'C': return 'J';
    case 'J': return 'C';
  }
  throw Error(std::string("bad transposition flag '") + t + "'");
}
char switch_conj(char t) {
  switch (t) {
    case 'N': return 'J';
    case 'T': return 'C';
    case 'C': return 'T';
    case 'J': return 'N';
  }
  throw Error(std::string("bad transposition flag '") + t + "'");
}

// op(Y) <- alpha op(B) op(X) + beta op(Y) with X, Y in internal numbering (gemm_dense,
// c_wrapping.hpp:302-366, side 'L' after the side 'R' rewrite): the operands are brought
// to client order, multiplied on the device, and returned.  Unlike the reference, X is not
// left conjugated on return for the 'C' / 'J' flags.
template <typename S>
void internal_product(hmat_matrix_t* m, char tb, char tx, char ty, S alpha, S beta, const S* X, S* Y, int nrhs) {
  if (tb != 'N' && tb != 'T' && tb != 'C') throw Error(std::string("bad transposition flag '") + tb + "'");
  if (tx != 'N' && tx != 'T' && tx != 'C' && tx != 'J') throw Error(std::string("bad transposition flag '") + tx + "'");
  const ClusterTree& rt = *m->rows_h->t;
  const ClusterTree& ct = *m->cols_h->t;
  const ClusterTree& in_t = !flag_trans(tb) ? ct : rt;
  const ClusterTree& out_t = !flag_trans(tb) ? rt : ct;
  const int nin = in_t.n, nout = out_t.n;
  std::vector<S> xc((size_t)nin * nrhs), yc((size_t)nout * nrhs);
  for (int q = 0; q < nrhs; ++q)
    for (int i = 0; i < nin; ++i) {
      S v = flag_trans(tx) ? X[q + (size_t)i * nrhs] : X[i + (size_t)q * nin];
      if (flag_conj(tx)) v = conj_s(v);
      xc[in_t.perm[i] + (size_t)q * nin] = v;
    }
  for (int q = 0; q < nrhs; ++q)
    for (int i = 0; i < nout; ++i) {
      S v = flag_trans(ty) ? Y[q + (size_t)i * nrhs] : Y[i + (size_t)q * nout];
      if (flag_conj(ty)) v = conj_s(v);
      yc[out_t.perm[i] + (size_t)q * nout] = v;
    }
  engine_of(m).gemv_host(tb, &alpha, xc.data(), &beta, yc.data(), nrhs);
  for (int q = 0; q < nrhs; ++q)
    for (int i = 0; i < nout; ++i) {
      S v = yc[out_t.perm[i] + (size_t)q * nout];
      if (flag_conj(ty)) v = conj_s(v);
      if (flag_trans(ty)) Y[q + (size_t)i * nrhs] = v;
      else Y[i + (size_t)q * nout] = v;
    }
}

template <int VT>
int gemm_dense_t(char trans_b, char trans_x, char side, const void* alpha, hmat_matrix_t* m, void* vec_x,
                 const void* beta, void* vec_y, int nrhs) {
  typedef typename HostScalar<VT>::type S;
  HB_TRY("gemm_dense", {
    if (!m || !alpha || !beta || (nrhs > 0 && (!vec_x || !vec_y))) throw Error("null argument");
    if (m->vt != VT) throw Error("matrix value type does not match this interface");
    S a = *(const S*)alpha, b = *(const S*)beta;
    char ty = 'N';
    if (side == 'R') {
      // Y <- alpha X op(B) + beta Y  <=>  Y^T <- alpha op(B)^T X^T + beta Y^T (or ^H)
      if (trans_b == 'C') {
        trans_b = 'N';
        trans_x = switch_conj(switch_trans(trans_x));
        ty = 'C';
        a = conj_s(a);
        b = conj_s(b);
      } else {
        trans_b = switch_trans(trans_b);
        trans_x = switch_trans(trans_x);
        ty = 'T';
      }
    } else if (side != 'L') {
      throw Error(std::string("bad side '") + side + "'");
    }
    if (nrhs > 0) internal_product<S>(m, trans_b, trans_x, ty, a, b, (const S*)vec_x, (S*)vec_y, nrhs);
  });
  return 0;
}

// gemm_scalar (c_wrapping.hpp:254-271): gemv in internal numbering.
template <int VT>
int gemm_scalar_t(char trans, void* alpha, hmat_matrix_t* m, void* x, void* beta, void* y, int nrhs) {
  typedef typename HostScalar<VT>::type S;
  HB_TRY("gemm_scalar", {
    if (!m || !alpha || !beta || (nrhs > 0 && (!x || !y))) throw Error("null argument");
    if (m->vt != VT) throw Error("matrix value type does not match this interface");
    if (nrhs > 0) internal_product<S>(m, trans, 'N', 'N', *(const S*)alpha, *(const S*)beta, (const S*)x, (S*)y, nrhs);
  });
  return 0;
}

// Fills out[r, c] (query positions) for every leaf that meets the sorted row and column
// queries (internal index, position), from the leaves' payloads.
template <typename S>
void fill_from_leaves(hmat_matrix_t* m, const std::vector<std::pair<int, int>>& rq,
                      const std::vector<std::pair<int, int>>& cq, S* out, size_t ld) {
  EngineBase& e = engine_of(m);
  if (!e.assembled) throw Error("matrix not assembled");
  const auto& L = m->bt.leaves;
  std::vector<S> buf;
  auto lo = [](const std::vector<std::pair<int, int>>& v, int x) {
    return (size_t)(std::lower_bound(v.begin(), v.end(), std::make_pair(x, -1)) - v.begin());
  };
  for (size_t i = 0; i < L.size(); ++i) {
    const LeafInfo& l = L[i];
    const size_t r0 = lo(rq, l.row_off), r1 = lo(rq, l.row_off + l.m);
    const size_t c0 = lo(cq, l.col_off), c1 = lo(cq, l.col_off + l.n);
    if (r0 == r1 || c0 == c1) continue;
    const int k = e.ranks[i];
    if (l.type == 1 && k <= 0) continue;  // zero block
    const size_t size = l.type == 0 ? (size_t)l.m * l.n : (size_t)k * (l.m + l.n);
    buf.resize(std::max<size_t>(size, 1));
    e.leaf_payload((int)i, buf.data());
    for (size_t a = r0; a < r1; ++a)
      for (size_t b = c0; b < c1; ++b) {
        const int ri = rq[a].first - l.row_off, cj = cq[b].first - l.col_off;
        S v;
        if (l.type == 0) {
          v = buf[ri + (size_t)l.m * cj];
        } else {
          v = S(0);
          const S* A = buf.data();
          const S* B = A + (size_t)l.m * k;
          for (int t = 0; t < k; ++t) v += A[ri + (size_t)l.m * t] * B[cj + (size_t)l.n * t];
        }
        out[rq[a].second + ld * cq[b].second] = v;
      }
  }
}

// get_block (c_wrapping.hpp:833-868, uncompressed_block.hpp): the dense block of rows
// [row_offset, +row_size) and columns [col_offset, +col_size) in internal numbering; the
// numbering arrays point into the cluster trees' internal -> client permutations.
template <int VT>
int get_block_t(struct hmat_get_values_context_t* ctx) {
  typedef typename HostScalar<VT>::type S;
  HB_TRY("get_block", {
    if (!ctx || !ctx->matrix || !ctx->values) throw Error("null argument");
    hmat_matrix_t* m = ctx->matrix;
    if (m->vt != VT) throw Error("matrix value type does not match this interface");
    ClusterTree& rt = *m->rows_h->t;
    ClusterTree& ct = *m->cols_h->t;
    if (ctx->row_offset < 0 || ctx->row_size < 0 || ctx->row_offset + ctx->row_size > rt.n || ctx->col_offset < 0 ||
        ctx->col_size < 0 || ctx->col_offset + ctx->col_size > ct.n)
      throw Error("block outside the matrix");
    const bool renumber = ctx->renumber_rows != 0;
    if (renumber && (ctx->row_offset != 0 || ctx->row_size != rt.n)) throw Error("Cannot renumber");
    std::vector<std::pair<int, int>> rq(ctx->row_size), cq(ctx->col_size);
    for (int i = 0; i < ctx->row_size; ++i) rq[i] = {ctx->row_offset + i, i};
    for (int j = 0; j < ctx->col_size; ++j) cq[j] = {ctx->col_offset + j, j};
    S* out = (S*)ctx->values;
    std::fill(out, out + (size_t)ctx->row_size * ctx->col_size, S(0));
    fill_from_leaves<S>(m, rq, cq, out, (size_t)ctx->row_size);
    if (renumber) {
      // restoreVectorOrder on the rows: row i of the block moves to client row perm[i]
      std::vector<S> tmp(ctx->row_size);
      for (int j = 0; j < ctx->col_size; ++j) {
        S* col = out + (size_t)j * ctx->row_size;
        for (int i = 0; i < ctx->row_size; ++i) tmp[rt.perm[i]] = col[i];
        std::copy(tmp.begin(), tmp.end(), col);
      }
    }
    ctx->row_indices = rt.perm.data() + ctx->row_offset;
    ctx->col_indices = ct.perm.data() + ctx->col_offset;
  });
  return 0;
}

// get_values (c_wrapping.hpp:871-890, uncompressed_values.hpp:82-95): entries for lists of
// rows and columns in natural numbering (1 to n); values[i + row_size j].
template <int VT>
int get_values_t(struct hmat_get_values_context_t* ctx) {
  typedef typename HostScalar<VT>::type S;
  HB_TRY("get_values", {
    if (!ctx || !ctx->matrix || !ctx->values || (ctx->row_size > 0 && !ctx->row_indices) ||
        (ctx->col_size > 0 && !ctx->col_indices))
      throw Error("null argument");
    hmat_matrix_t* m = ctx->matrix;
    if (m->vt != VT) throw Error("matrix value type does not match this interface");
    const ClusterTree& rt = *m->rows_h->t;
    const ClusterTree& ct = *m->cols_h->t;
    std::vector<std::pair<int, int>> rq(ctx->row_size), cq(ctx->col_size);
    for (int i = 0; i < ctx->row_size; ++i) {
      const int q = ctx->row_indices[i];
      if (q < 1 || q > rt.n) throw Error("row index outside 1..n");
      rq[i] = {rt.rev[q - 1], i};
    }
    for (int j = 0; j < ctx->col_size; ++j) {
      const int q = ctx->col_indices[j];
      if (q < 1 || q > ct.n) throw Error("column index outside 1..n");
      cq[j] = {ct.rev[q - 1], j};
    }
    std::sort(rq.begin(), rq.end());
    std::sort(cq.begin(), cq.end());
    S* out = (S*)ctx->values;
    std::fill(out, out + (size_t)ctx->row_size * ctx->col_size, S(0));
    fill_from_leaves<S>(m, rq, cq, out, (size_t)ctx->row_size);
  });
  return 0;
}
int u_add_identity(hmat_matrix_t*, void*) { return unsupported("add_identity"); }
int u_get_profile(hmat_matrix_t*, hmat_profile_t*) { return unsupported("get_profile"); }
int u_get_ratio(hmat_matrix_t*, hmat_FPCompressionRatio_t*) { return unsupported("get_ratio"); }
int u_fpcompress(hmat_matrix_t*) { return unsupported("FPcompress"); }
int u_fpdecompress(hmat_matrix_t*) { return unsupported("FPdecompress"); }
hmat_fp_settings_t u_get_fp(hmat_matrix_t*) {
  unsupported("GetFPCompressionSettings");
  hmat_fp_settings_t s;
  memset(&s, 0, sizeof(s));
  return s;
}
int u_set_fp(hmat_matrix_t*, hmat_fp_settings_t) { return unsupported("SetFPCompressionSettings"); }
int u_set_fp_params(hmat_matrix_t*, float, int, hmat_FPcompress_t, bool, bool) {
  return unsupported("SetFPCompressionSettingsParams");
}
int u_dump_info(hmat_matrix_t*, char*) { return unsupported("dump_info"); }
int u_set_cluster_trees(hmat_matrix_t*, const hmat_cluster_tree_t*, const hmat_cluster_tree_t*) {
  return unsupported("set_cluster_trees");
}
int u_extract_diagonal(hmat_matrix_t*, void*, int) { return unsupported("extract_diagonal"); }
int u_solve_lower(hmat_matrix_t*, int, void*, int) { return unsupported("solve_lower_triangular"); }
int u_solve_lower_dense(hmat_matrix_t*, int, void*, int) { return unsupported("solve_lower_triangular_dense"); }

int u_walk(hmat_matrix_t*, hmat_procedure_t*) { return unsupported("walk"); }
int u_apply_on_leaf(hmat_matrix_t*, const hmat_leaf_procedure_t*) { return unsupported("apply_on_leaf"); }
// ---- write_struct / read_struct / write_data / read_data (c_wrapping.hpp:921-946) ----
// Structure: this library's own stream format (native byte order), through the caller's
// hmat_iostream (the reference's structure stream carries its internal node tree and the
// cluster data classes, so structure streams are not exchangeable):
//   struct: "HB2S", version, value type, rows tree, cols-tree flag (0: same as rows) [+ cols
//           tree], leaf count, leaves (row node, col node, row offset, m, col offset, n, type),
//           number of block clusters, low-rank epsilon, end mark "HB2E"
//   tree:   n, points (3 n doubles, client numbering), permutation (internal -> client),
//           node count, nodes (offset, size, children, child count, depth, bounding box),
//           tree-leaf count, tree leaves
// Data: the reference's own data stream (MatrixDataMarshaller / MatrixDataUnmarshaller,
// serialization.cpp:248-309 and 318-394), so that a matrix written by one library loads into
// a matrix of the same partition built by the other: the non-empty leaves in depth-first order
// (the leaf table's order), each as
//   Rk leaf:   int rank; if rank > 0: A (m x k) then B (n x k), column-major scalars of the
//              matrix's type, then the orthogonality flags of A and B (two ints, written 0)
//   full leaf: int header (bit 0: null block, no data; bit 1: pivots; bit 2: diagonal: the
//              factorised forms, refused here), then F (m x n, column-major)
// The data stream has no header of its own: a matrix whose partition differs from the writer's
// reads garbage, which the reader refuses where it can (ranks outside [0, min(m, n)], unknown
// headers, a stream cut short).
const int kStreamVersion = 1;
struct StreamOut {
  hmat_iostream f;
  void* ud;
  template <typename X>
  void val(X v) { f(&v, sizeof v, ud); }
  void bytes(const void* p, size_t n) {
    if (n) f(const_cast<void*>(p), n, ud);
  }
};
struct StreamIn {
  hmat_iostream f;
  void* ud;
  template <typename X>
  X val() {
    X v;
    f(&v, sizeof v, ud);
    return v;
  }
  void bytes(void* p, size_t n) {
    if (n) f(p, n, ud);
  }
};
void write_magic(StreamOut& o, char kind) {
  const char mg[4] = {'H', 'B', '2', kind};
  o.bytes(mg, 4);
  o.val<int>(kStreamVersion);
}
// Every stream ends with "HB2E": a stream cut short (or padded) is refused.
void write_end(StreamOut& o) {
  const char mg[4] = {'H', 'B', '2', 'E'};
  o.bytes(mg, 4);
}
void read_end(StreamIn& in) {
  char mg[4];
  in.bytes(mg, 4);
  if (mg[0] != 'H' || mg[1] != 'B' || mg[2] != '2' || mg[3] != 'E') throw Error("corrupt stream (no end mark)");
}
void read_magic(StreamIn& in, char kind) {
  char mg[4];
  in.bytes(mg, 4);
  if (mg[0] != 'H' || mg[1] != 'B' || mg[2] != '2' || mg[3] != kind) throw Error("not a B200 engine stream");
  if (in.val<int>() != kStreamVersion) throw Error("unsupported stream version");
}
void write_tree(StreamOut& o, const ClusterTree& t) {
  o.val<int>(t.n);
  o.bytes(t.pts.data(), t.pts.size() * sizeof(double));
  o.bytes(t.perm.data(), t.perm.size() * sizeof(int));
  o.val<int>((int)t.nodes.size());
  for (const ClusterNode& c : t.nodes) {
    o.val<int>(c.offset);
    o.val<int>(c.size);
    o.val<int>(c.child[0]);
    o.val<int>(c.child[1]);
    o.val<int>(c.nchild);
    o.val<int>(c.depth);
    o.bytes(c.bb, sizeof c.bb);
  }
  o.val<int>((int)t.leaf_nodes.size());
  o.bytes(t.leaf_nodes.data(), t.leaf_nodes.size() * sizeof(int));
}
std::unique_ptr<ClusterTree> read_tree(StreamIn& in) {
  auto t = std::make_unique<ClusterTree>();
  t->n = in.val<int>();
  if (t->n < 0) throw Error("corrupt stream (tree size)");
  t->pts.resize((size_t)t->n * 3);
  in.bytes(t->pts.data(), t->pts.size() * sizeof(double));
  t->perm.resize(t->n);
  in.bytes(t->perm.data(), t->perm.size() * sizeof(int));
  t->rev.assign(t->n, -1);
  for (int i = 0; i < t->n; ++i) {
    if (t->perm[i] < 0 || t->perm[i] >= t->n || t->rev[t->perm[i]] != -1) throw Error("corrupt stream (permutation)");
    t->rev[t->perm[i]] = i;
  }
  const int nn = in.val<int>();
  if (nn < 0) throw Error("corrupt stream (node count)");
  t->nodes.resize(nn);
  for (ClusterNode& c : t->nodes) {
    c.offset = in.val<int>();
    c.size = in.val<int>();
    c.child[0] = in.val<int>();
    c.child[1] = in.val<int>();
    c.nchild = in.val<int>();
    c.depth = in.val<int>();
    in.bytes(c.bb, sizeof c.bb);
    if (c.offset < 0 || c.size < 0 || c.offset + c.size > t->n || c.child[0] >= nn || c.child[1] >= nn)
      throw Error("corrupt stream (node)");
  }
  const int nl = in.val<int>();
  if (nl < 0) throw Error("corrupt stream (tree leaves)");
  t->leaf_nodes.resize(nl);
  in.bytes(t->leaf_nodes.data(), (size_t)nl * sizeof(int));
  return t;
}

void c_write_struct(hmat_matrix_t* m, hmat_iostream f, void* ud) {
  try {
    if (!m || !f) throw Error("null argument");
    StreamOut o{f, ud};
    write_magic(o, 'S');
    o.val<int>(m->vt);
    write_tree(o, *m->rows_h->t);
    const bool same = m->cols_h == m->rows_h;
    o.val<int>(same ? 0 : 1);
    if (!same) write_tree(o, *m->cols_h->t);
    o.val<int>((int)m->bt.leaves.size());
    for (const LeafInfo& l : m->bt.leaves) {
      const int v[7] = {l.row_node, l.col_node, l.row_off, l.m, l.col_off, l.n, l.type};
      o.bytes(v, sizeof v);
    }
    o.val<int>(m->bt.nr_block_clusters);
    o.val<double>(m->low_rank_eps);
    write_end(o);
  } catch (const std::exception& e) {
    fail("write_struct", e.what());
  }
}

template <int VT>
hmat_matrix_t* c_read_struct(hmat_iostream f, void* ud) {
  std::unique_ptr<hmat_matrix_t> m;
  std::unique_ptr<hmat_cluster_tree_t> rt, ct;
  try {
    if (!f) throw Error("null argument");
    StreamIn in{f, ud};
    read_magic(in, 'S');
    if (in.val<int>() != VT) throw Error("Type mismatch between the stream and this interface");
    rt.reset(new hmat_cluster_tree_t());
    rt->t = read_tree(in);
    if (in.val<int>() != 0) {
      ct.reset(new hmat_cluster_tree_t());
      ct->t = read_tree(in);
    }
    m.reset(new hmat_matrix_t());
    m->vt = VT;
    const int nl = in.val<int>();
    if (nl < 0) throw Error("corrupt stream (leaf count)");
    const int nr = rt->t->n, nc = ct ? ct->t->n : nr;
    m->bt.leaves.resize(nl);
    for (LeafInfo& l : m->bt.leaves) {
      int v[7];
      in.bytes(v, sizeof v);
      l.row_node = v[0];
      l.col_node = v[1];
      l.row_off = v[2];
      l.m = v[3];
      l.col_off = v[4];
      l.n = v[5];
      l.type = v[6];
      if (l.row_off < 0 || l.m < 0 || l.row_off + l.m > nr || l.col_off < 0 || l.n < 0 || l.col_off + l.n > nc ||
          (l.type != 0 && l.type != 1))
        throw Error("corrupt stream (leaf)");
    }
    m->bt.nr_block_clusters = in.val<int>();
    m->low_rank_eps = in.val<double>();
    read_end(in);
    m->rows_h = rt.release();
    m->cols_h = ct ? ct.release() : m->rows_h;
    m->own_rows = m->own_cols = true;
    return m.release();
  } catch (const std::exception& e) {
    fail("read_struct", e.what());
    return nullptr;
  }
}

template <int VT>
void c_write_data(hmat_matrix_t* m, hmat_iostream f, void* ud) {
  typedef typename HostScalar<VT>::type S;
  try {
    if (!m || !f) throw Error("null argument");
    if (m->vt != VT) throw Error("matrix value type does not match this interface");
    EngineBase& e = engine_of(m);
    if (!e.assembled) throw Error("write_data needs an assembled matrix");
    const int nl = (int)m->bt.leaves.size();
    StreamOut o{f, ud};
    std::vector<S> buf;
    for (int i = 0; i < nl; ++i) {
      const LeafInfo& l = m->bt.leaves[i];
      if (l.m == 0 || l.n == 0) continue;  // void blocks are not written (serialization.cpp:293-296)
      const int k = l.type == 0 ? 0 : std::max(e.ranks[i], 0);
      o.val<int>(l.type == 0 ? 0 : k);
      const size_t size = l.type == 0 ? (size_t)l.m * l.n : (size_t)k * (l.m + l.n);
      if (size) {
        buf.resize(size);
        e.leaf_payload(i, buf.data());
        o.bytes(buf.data(), size * sizeof(S));
      }
      if (l.type == 1 && k > 0) {
        o.val<int>(0);
        o.val<int>(0);
      }
    }
  } catch (const std::exception& ex) {
    fail("write_data", ex.what());
  }
}

template <int VT>
void c_read_data(hmat_matrix_t* m, hmat_iostream f, void* ud) {
  typedef typename HostScalar<VT>::type S;
  try {
    if (!m || !f) throw Error("null argument");
    if (m->vt != VT) throw Error("matrix value type does not match this interface");
    StreamIn in{f, ud};
    const int nl = (int)m->bt.leaves.size();
    std::vector<int> rk(nl, 0);
    std::vector<S> payload;
    for (int i = 0; i < nl; ++i) {
      const LeafInfo& l = m->bt.leaves[i];
      if (l.m == 0 || l.n == 0) {
        rk[i] = l.type == 0 ? -1 : 0;
        continue;
      }
      const int header = in.val<int>();
      if (l.type == 1) {
        if (header < 0 || header > std::min(l.m, l.n))
          throw Error("corrupt stream or another partition (Rk leaf " + std::to_string(i) + " with rank " +
                      std::to_string(header) + ")");
        rk[i] = header;
        if (header > 0) {
          const size_t at = payload.size(), size = (size_t)header * (l.m + l.n);
          payload.resize(at + size);
          in.bytes(payload.data() + at, size * sizeof(S));
          in.val<int>();  // orthogonality of A and B: not used by this library
          in.val<int>();
        }
      } else {
        rk[i] = -1;
        if (header & ~7) throw Error("corrupt stream or another partition (full leaf " + std::to_string(i) + ")");
        if (header & 6) throw Error("factorised full blocks (pivots or diagonal) are outside the B200 engine");
        const size_t at = payload.size(), size = (size_t)l.m * l.n;
        payload.resize(at + size, S(0));
        if (!(header & 1)) in.bytes(payload.data() + at, size * sizeof(S));  // bit 0: a null block
      }
    }
    // the reference's reader ends with a read of 0 bytes (serialization.cpp:390-391)
    S dummy;
    f(&dummy, 0, ud);
    payload.resize(std::max<size_t>(payload.size(), 1));
    engine_of(m).load_leaves(rk.data(), payload.data());
  } catch (const std::exception& e) {
    fail("read_data", e.what());
  }
}
void u_set_progressbar(hmat_matrix_t*, hmat_progress_t*) {}
int u_extract_diagonal_block(hmat_matrix_t*, int, void*) { return unsupported("extract_diagonal_block"); }

template <int VT, typename T>
void fill_table(hmat_interface_t* i) {
  i->create_empty_hmatrix_admissibility = create_empty_t<VT>;
  i->own_cluster_trees = own_cluster_trees;
  i->set_low_rank_epsilon = set_low_rank_epsilon;
  i->assemble_generic = assemble_generic;
  i->copy = u_copy;
  i->copy_struct = u_copy_struct;
  i->norm = u_norm;
  i->logdet = u_logdet;
  i->inverse = u_inverse;
  i->factorize_generic = u_factorize;
  i->destroy = destroy;
  i->get_child = u_get_child;
  i->destroy_child = u_destroy_child;
  i->solve_generic = u_solve_generic;
  i->solve_mat = u_solve_mat;
  i->solve_systems = u_solve_systems;
  i->solve_dense = u_solve_dense;
  i->transpose = u_transpose;
  i->scale = u_scale;
  i->truncate = c_truncate;
  i->vector_reorder = vector_reorder_t<T>;
  i->vector_restore = vector_restore_t<T>;
  i->gemm = u_gemm;
  i->axpy = u_axpy;
  i->trsm = u_trsm;
  i->gemv = gemv_t<VT>;
  i->gemm_scalar = gemm_scalar_t<VT>;
  i->full_gemm = u_full_gemm;
  i->gemm_dense = gemm_dense_t<VT>;
  i->add_identity = u_add_identity;
  i->init = init_fn;
  i->finalize = finalize_fn;
  i->get_info = get_info;
  i->get_profile = u_get_profile;
  i->get_ratio = u_get_ratio;
  i->FPcompress = u_fpcompress;
  i->FPdecompress = u_fpdecompress;
  i->GetFPCompressionSettings = u_get_fp;
  i->SetFPCompressionSettings = u_set_fp;
  i->SetFPCompressionSettingsParams = u_set_fp_params;
  i->dump_info = u_dump_info;
  i->get_cluster_trees = get_cluster_trees;
  i->set_cluster_trees = u_set_cluster_trees;
  i->extract_diagonal = u_extract_diagonal;
  i->solve_lower_triangular = u_solve_lower;
  i->solve_lower_triangular_dense = u_solve_lower_dense;
  i->get_block = get_block_t<VT>;
  i->get_values = get_values_t<VT>;
  i->walk = u_walk;
  i->apply_on_leaf = u_apply_on_leaf;
  i->internal = nullptr;
  i->read_struct = c_read_struct<VT>;
  i->write_struct = c_write_struct;
  i->read_data = c_read_data<VT>;
  i->write_data = c_write_data<VT>;
  i->set_progressbar = u_set_progressbar;
  i->extract_diagonal_block = u_extract_diagonal_block;
}

}  // namespace

extern "C" {

hmat_clustering_algorithm_t* hmat_create_clustering_median(void) { return new hmat_clustering_algorithm(); }

hmat_clustering_algorithm_t* hmat_create_clustering_max_dof(const hmat_clustering_algorithm_t* algo, int max_dof) {
  if (!algo) return nullptr;
  hmat_clustering_algorithm* r = new hmat_clustering_algorithm(*algo);
  r->a.max_leaf = max_dof;
  return r;
}

void hmat_delete_clustering(hmat_clustering_algorithm_t* algo) { delete algo; }

void hmat_set_clustering_divider(hmat_clustering_algorithm_t* algo, int divider) {
  if (algo) algo->a.divider = divider;
}

hmat_cluster_tree_t* hmat_create_cluster_tree(double* coord, int dimension, int size,
                                              hmat_clustering_algorithm_t* algo) {
  try {
    if (!coord || !algo) throw Error("null argument");
    if (dimension != 3) throw Error("the B200 engine clusters 3-D points only");
    if (algo->a.divider != 2) throw Error("only bisection (divider 2) is supported");
    const int leaf = algo->a.max_leaf >= 0 ? algo->a.max_leaf : g_settings.maxLeafSize;
    hmat_cluster_tree_t* t = new hmat_cluster_tree_t();
    t->t = build_cluster_tree(coord, size, leaf);
    return t;
  } catch (const std::exception& e) {
    fail("hmat_create_cluster_tree", e.what());
    return nullptr;
  }
}

void hmat_delete_cluster_tree(const hmat_cluster_tree_t* tree) { delete tree; }

int hmat_tree_nodes_count(const hmat_cluster_tree_t* tree) { return tree ? (int)tree->t->nodes.size() : 0; }

int hmat_cluster_get_info(hmat_cluster_tree_t* tree, hmat_cluster_info_t* info) {
  if (!tree || !info) return fail("hmat_cluster_get_info", "null argument");
  info->spatial_dimension = 3;
  info->dimension = tree->t->n;
  info->nr_tree_nodes = tree->t->nodes.size();
  return 0;
}

const int* hmat_cluster_get_indices(const hmat_cluster_tree_t* tree) { return tree ? tree->t->perm.data() : nullptr; }

void hmat_init_admissibility_param(hmat_admissibility_param_t* p) {
  if (!p) return;
  p->eta = 2;
  p->ratio = 0.0;
  p->max_width = (size_t)-1;
  p->scale = -1;
}

hmat_admissibility_t* hmat_create_admissibility(hmat_admissibility_param_t* p) {
  if (!p) return nullptr;
  hmat_admissibility_condition* c = new hmat_admissibility_condition();
  c->a.eta = p->eta;
  c->a.ratio = p->ratio;
  c->a.max_width = p->max_width;
  return c;
}

void hmat_update_admissibility(hmat_admissibility_t* cond, hmat_admissibility_param_t* p) {
  if (!cond || !p) return;
  cond->a.eta = p->eta;
  cond->a.ratio = p->ratio;
  cond->a.max_width = p->max_width;
}

hmat_admissibility_t* hmat_create_admissibility_standard(double eta) {
  hmat_admissibility_condition* c = new hmat_admissibility_condition();
  c->a.eta = eta;
  return c;
}

void hmat_delete_admissibility(hmat_admissibility_t* cond) { delete cond; }

static hmat_compression_algorithm_t* make_compression(hmat_compress_t m, double eps) {
  hmat_compression_algorithm_t* c = new hmat_compression_algorithm_t();
  c->method = m;
  c->eps = eps;
  return c;
}
hmat_compression_algorithm_t* hmat_create_compression_aca_plus(double e) {
  return make_compression(hmat_compress_aca_plus, e);
}
hmat_compression_algorithm_t* hmat_create_compression_aca_partial(double e) {
  return make_compression(hmat_compress_aca_partial, e);
}
hmat_compression_algorithm_t* hmat_create_compression_svd(double e) { return make_compression(hmat_compress_svd, e); }
hmat_compression_algorithm_t* hmat_create_compression_aca_full(double e) {
  return make_compression(hmat_compress_aca_full, e);
}
hmat_compression_algorithm_t* hmat_create_compression_aca_random(double e) {
  return make_compression(hmat_compress_aca_random, e);
}
hmat_compression_algorithm_t* hmat_create_compression_rrqr(double e) {
  return make_compression(hmat_compress_rrqr, e);
}
void hmat_delete_compression(const hmat_compression_algorithm_t* algo) { delete algo; }

void hmat_assemble_context_init(hmat_assemble_context_t* c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  c->factorization = hmat_factorization_none;
}

void hmat_factorization_context_init(hmat_factorization_context_t* c) {
  if (!c) return;
  c->factorization = hmat_factorization_lu;
  c->progress = nullptr;
}

void hmat_solve_context_init(struct hmat_solve_context_t* c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
}

hmat_progress_t* hmat_default_progress(void) {
  static hmat_progress_t p = {0, 0, nullptr, nullptr};
  return &p;
}

void hmat_init_default_interface(hmat_interface_t* i, hmat_value_t type) {
  if (!i) return;
  memset(i, 0, sizeof(*i));
  i->value_type = type;
  switch (type) {
    case HMAT_SIMPLE_PRECISION: fill_table<0, float>(i); break;
    case HMAT_DOUBLE_PRECISION: fill_table<1, double>(i); break;
    case HMAT_SIMPLE_COMPLEX: fill_table<2, std::complex<float>>(i); break;
    case HMAT_DOUBLE_COMPLEX: fill_table<3, std::complex<double>>(i); break;
    default: fail("hmat_init_default_interface", "unknown value type");
  }
}

void hmat_get_parameters(hmat_settings_t* s) {
  if (s) *s = g_settings;
}

int hmat_set_parameters(hmat_settings_t* s) {
  if (!s) return fail("hmat_set_parameters", "null settings");
  g_settings = *s;
  return 0;
}

const char* hmat_get_version(void) { return "1.11.1-b200"; }

// ---------------------------------------------------------------------------------

void* hmat_b200_create_assembly(const hmat_b200_kernel_t* k, const double* coord, int n) {
  if (!k || !coord || n <= 0) {
    fail("hmat_b200_create_assembly", "bad argument");
    return nullptr;
  }
  if (k->kind < HMAT_B200_LAPLACE_REG || k->kind > HMAT_B200_HELMHOLTZ_REG) {
    fail("hmat_b200_create_assembly", "unknown kernel kind");
    return nullptr;
  }
  if (k->kind == HMAT_B200_EXP_COV && !(k->ell > 0)) {
    fail("hmat_b200_create_assembly", "exp_cov needs ell > 0");
    return nullptr;
  }
  AssemblyObj* a = new AssemblyObj();
  a->d.kp.kind = (int)k->kind;
  a->d.kp.delta = k->delta;
  a->d.kp.ell = k->ell;
  a->d.kp.nugget = k->nugget;
  a->d.kp.wavenumber = k->wavenumber;
  a->d.pts.assign(coord, coord + 3 * (size_t)n);
  return a;
}

void* hmat_b200_create_assembly_strata(const hmat_b200_kernel_t* k, const double* coord, int n, int nstrata,
                                       const double* param, const double* weight) {
  if (!k || !coord || n <= 0 || !param || !weight || nstrata < 1 || nstrata > kMaxStrata) {
    fail("hmat_b200_create_assembly_strata", "bad argument (1 to 8 strata, parameters and weights)");
    return nullptr;
  }
  for (int q = 0; q < nstrata; ++q) {
    if (k->kind == HMAT_B200_EXP_COV && !(param[q] > 0)) {
      fail("hmat_b200_create_assembly_strata", "exp_cov strata need correlation lengths > 0");
      return nullptr;
    }
    if (!std::isfinite(param[q]) || !std::isfinite(weight[q])) {
      fail("hmat_b200_create_assembly_strata", "non-finite stratum parameter or weight");
      return nullptr;
    }
  }
  hmat_b200_kernel_t k1 = *k;
  if (k1.kind == HMAT_B200_EXP_COV) k1.ell = param[0];  // the plain kernel's own check
  AssemblyObj* a = (AssemblyObj*)hmat_b200_create_assembly(&k1, coord, n);
  if (!a) return nullptr;
  a->d.kp.ell = k->ell;
  a->d.strata.assign(param, param + nstrata);
  a->d.strata.insert(a->d.strata.end(), weight, weight + nstrata);
  return a;
}

void hmat_b200_delete_assembly(void* a) {
  AssemblyObj* o = (AssemblyObj*)a;
  if (o && o->magic == kAssemblyMagic) {
    o->magic = 0;
    delete o;
  }
}

int hmat_b200_gemv_device(hmat_matrix_t* m, char trans, const void* alpha, const void* x, const void* beta, void* y,
                          int nrhs, void* stream) {
  HB_TRY("hmat_b200_gemv_device", {
    if (!m || !alpha || !beta || (nrhs > 0 && (!x || !y))) throw Error("null argument");
    engine_of(m).gemv_device(trans, alpha, x, beta, y, nrhs, (cudaStream_t)stream);
  });
  return 0;
}

int hmat_b200_gemv_status(hmat_matrix_t* m, void* stream, int* failed) {
  HB_TRY("hmat_b200_gemv_status", {
    if (!m || !failed) throw Error("null argument");
    if (!m->engine || !m->engine->assembled) throw Error("matrix is not assembled");
    *failed = m->engine->gemv_status((cudaStream_t)stream);
  });
  return 0;
}

// ---- batches of independent matrices ----
// The batch is the block-diagonal matrix of its members: their cluster trees side by side (row
// and column numbering offset by the rows before each member), their leaves in member order.
// It is an ordinary hmat_matrix_t for every other entry point (one assembly and one product
// for all members, one launch per phase), and owns its combined tree.
hmat_matrix_t* hmat_b200_batch_create(hmat_matrix_t* const* matrices, int count) {
  try {
    if (!matrices || count <= 0) throw Error("bad argument");
    std::unique_ptr<hmat_cluster_tree_t> tree(new hmat_cluster_tree_t());
    tree->t.reset(new ClusterTree());
    ClusterTree& t = *tree->t;
    std::unique_ptr<hmat_matrix_t> b(new hmat_matrix_t());
    b->vt = matrices[0] ? matrices[0]->vt : 1;
    b->low_rank_eps = matrices[0] ? matrices[0]->low_rank_eps : 1e-4;
    b->batch_rows.push_back(0);
    b->batch_leaves.push_back(0);
    for (int i = 0; i < count; ++i) {
      const hmat_matrix_t* m = matrices[i];
      if (!m) throw Error("null member matrix");
      if (!m->batch_rows.empty()) throw Error("a batch cannot be a member of a batch");
      if (m->vt != b->vt) throw Error("the members of a batch must have one value type");
      if (m->rows_h != m->cols_h) throw Error("batch members must be built on one cluster tree (rows = columns)");
      if (m->low_rank_eps != b->low_rank_eps) throw Error("the members of a batch must have one low-rank epsilon");
      const ClusterTree& s = *m->rows_h->t;
      const int base = t.n, nbase = (int)t.nodes.size();
      t.pts.insert(t.pts.end(), s.pts.begin(), s.pts.end());
      for (int v : s.perm) t.perm.push_back(v + base);
      for (int v : s.rev) t.rev.push_back(v + base);
      for (ClusterNode c : s.nodes) {
        c.offset += base;
        for (int& ch : c.child)
          if (ch >= 0) ch += nbase;
        t.nodes.push_back(c);
      }
      for (int l : s.leaf_nodes) t.leaf_nodes.push_back(l + nbase);
      t.n += s.n;
      for (LeafInfo l : m->bt.leaves) {
        l.row_node += nbase;
        l.col_node += nbase;
        l.row_off += base;
        l.col_off += base;
        b->bt.leaves.push_back(l);
      }
      b->bt.nr_block_clusters += m->bt.nr_block_clusters;
      b->batch_rows.push_back(t.n);
      b->batch_leaves.push_back((int)b->bt.leaves.size());
    }
    b->rows_h = b->cols_h = tree.release();
    b->own_rows = true;
    return b.release();
  } catch (const std::exception& e) {
    fail("hmat_b200_batch_create", e.what());
    return nullptr;
  }
}

int hmat_b200_batch_offsets(hmat_matrix_t* b, int* row_base, int* leaf_base) {
  if (!b || b->batch_rows.empty()) return fail("hmat_b200_batch_offsets", "not a batch");
  for (size_t i = 0; i < b->batch_rows.size(); ++i) {
    if (row_base) row_base[i] = b->batch_rows[i];
    if (leaf_base) leaf_base[i] = b->batch_leaves[i];
  }
  return 0;
}

int hmat_b200_batch_assemble(hmat_matrix_t* b, void* const* assemblies, const hmat_compression_algorithm_t* comp) {
  HB_TRY("hmat_b200_batch_assemble", {
    if (!b || !assemblies || !comp) throw Error("null argument");
    const int count = (int)b->batch_rows.size() - 1;
    if (count <= 0) throw Error("not a batch");
    int method;
    switch (comp->method) {
      case hmat_compress_aca_plus: method = 0; break;
      case hmat_compress_aca_partial: method = 1; break;
      default: throw Error("only ACA+ and partial-ACA compression are implemented by the B200 engine");
    }
    AssemblyDesc d;
    bool uniform = true;
    std::vector<double> param;
    for (int i = 0; i < count; ++i) {
      const AssemblyObj* a = (const AssemblyObj*)assemblies[i];
      if (!a || a->magic != kAssemblyMagic) throw Error("member assembly is not a descriptor from hmat_b200_create_assembly");
      const int n = b->batch_rows[i + 1] - b->batch_rows[i];
      if ((long long)a->d.pts.size() != 3LL * n) throw Error("member assembly has another point count than its matrix");
      const KernelParams& k = a->d.kp;
      if (!a->d.strata.empty()) throw Error("multi-strata kernels are not supported in batches");
      if (i == 0) d.kp = k;
      if (k.kind != d.kp.kind) throw Error("the members of a batch must share the kernel kind");
      if (k.nugget != d.kp.nugget) throw Error("the members of a batch must share the covariance nugget");
      if (k.kind == kHelmholtzReg && k.delta != d.kp.delta)
        throw Error("the members of a Helmholtz batch must share the regularisation");
      const double own = k.kind == kExpCov ? k.ell : (k.kind == kLaplaceReg ? k.delta : k.wavenumber);
      const double first = d.kp.kind == kExpCov ? d.kp.ell : (d.kp.kind == kLaplaceReg ? d.kp.delta : d.kp.wavenumber);
      if (own != first) uniform = false;
      d.pts.insert(d.pts.end(), a->d.pts.begin(), a->d.pts.end());
      param.insert(param.end(), (size_t)n, own);
    }
    if (!uniform) d.param.swap(param);  // each member's own parameter, point by point
    engine_of(b).assemble(d, method, comp->eps, b->low_rank_eps, g_settings.compressionMinLeafSize);
  });
  return 0;
}

int hmat_b200_leaf_count(hmat_matrix_t* m) { return m ? (int)m->bt.leaves.size() : -1; }

int hmat_b200_leaf_table(hmat_matrix_t* m, int* out) {
  if (!m || !out) return fail("hmat_b200_leaf_table", "null argument");
  const auto& L = m->bt.leaves;
  for (size_t i = 0; i < L.size(); ++i) {
    out[6 * i + 0] = L[i].row_off;
    out[6 * i + 1] = L[i].m;
    out[6 * i + 2] = L[i].col_off;
    out[6 * i + 3] = L[i].n;
    out[6 * i + 4] = L[i].type;
    out[6 * i + 5] = leaf_rank(m, i);
  }
  return 0;
}

long long hmat_b200_leaf_payload(hmat_matrix_t* m, int leaf, void* out) {
  try {
    if (!m || !out) throw Error("null argument");
    return engine_of(m).leaf_payload(leaf, out);
  } catch (const std::exception& e) {
    fail("hmat_b200_leaf_payload", e.what());
    return -1;
  }
}

int hmat_b200_payload_layout(hmat_matrix_t* m, long long* offsets, long long* total) {
  HB_TRY("hmat_b200_payload_layout", {
    if (!m) throw Error("null matrix");
    if (!engine_of(m).assembled) throw Error("matrix is not assembled");
    m->engine->payload_layout(offsets, total);
  });
  return 0;
}

int hmat_b200_leaf_gradients(hmat_matrix_t* m, const void* x, const void* r, int nrhs, void* grad, int accumulate,
                             void* stream) {
  HB_TRY("hmat_b200_leaf_gradients", {
    if (!m || !x || !r || !grad) throw Error("null argument");
    engine_of(m).leaf_gradients(x, r, nrhs, grad, accumulate != 0, (cudaStream_t)stream);
  });
  return 0;
}

int hmat_b200_gemv_adjoint(hmat_matrix_t* m, const void* x, const void* r, int nrhs, void* dx, void* grad,
                           int accumulate, void* stream) {
  HB_TRY("hmat_b200_gemv_adjoint", {
    if (!m || !x || !r || !dx || !grad) throw Error("null argument");
    engine_of(m).gemv_adjoint(x, r, nrhs, dx, grad, accumulate != 0, (cudaStream_t)stream);
  });
  return 0;
}

int hmat_b200_gemv_profile(hmat_matrix_t* m, char trans, const void* x_dev, void* y_dev, int nrhs, double* ms3,
                           double* bytes3) {
  HB_TRY("hmat_b200_gemv_profile", {
    if (!m || !x_dev || !y_dev || !ms3 || !bytes3) throw Error("null argument");
    engine_of(m).profile_gemv(trans, x_dev, y_dev, nrhs, ms3, bytes3);
  });
  return 0;
}

int hmat_b200_gemv_launches(hmat_matrix_t* m, char trans, int nrhs) {
  try {
    if (!m || nrhs < 1) throw Error("bad argument");
    return engine_of(m).gemv_launches(trans, nrhs);
  } catch (const std::exception& e) {
    fail("hmat_b200_gemv_launches", e.what());
    return -1;
  }
}

int hmat_b200_phase_times(hmat_matrix_t* m, double* out4) {
  if (!m || !out4) return fail("hmat_b200_phase_times", "null argument");
  for (int i = 0; i < 4; ++i) out4[i] = m->engine ? m->engine->times_ms[i] : 0.0;
  return 0;
}

int hmat_b200_aca_shapes(hmat_matrix_t* m, int* shape4, int* tuned4, double* rate20) {
  if (!m || !shape4 || !tuned4 || !rate20) return fail("hmat_b200_aca_shapes", "null argument");
  for (int b = 0; b < 4; ++b) {
    shape4[b] = m->engine ? m->engine->aca_shape[b] : -1;
    tuned4[b] = m->engine ? m->engine->aca_tuned[b] : 0;
    for (int s = 0; s < 5; ++s) rate20[5 * b + s] = m->engine ? m->engine->aca_rate[b][s] : 0.0;
  }
  return 0;
}

int hmat_b200_gemv_tuning(hmat_matrix_t* m, int* choice2, int* how, double* ms5) {
  if (!m || !choice2 || !how || !ms5) return fail("hmat_b200_gemv_tuning", "null argument");
  if (!m->engine || !m->engine->assembled) return fail("hmat_b200_gemv_tuning", "matrix is not assembled");
  choice2[0] = m->engine->gemv_choice[0];
  choice2[1] = m->engine->gemv_choice[1];
  *how = m->engine->gemv_tuned;
  for (int i = 0; i < 5; ++i) ms5[i] = m->engine->gemv_rate[i];
  return 0;
}

const char* hmat_b200_last_error(void) { return g_last_error.c_str(); }
void hmat_b200_clear_last_error(void) { g_last_error.clear(); }

}  // extern "C"

// Internal helpers for the other translation units of the library (not exported).
namespace hmatb200 {
EngineBase* existing_engine(hmat_matrix_t* m) { return m ? m->engine.get() : nullptr; }
int report_failure(const char* where, const std::string& msg) { return fail(where, msg); }
}  // namespace hmatb200
