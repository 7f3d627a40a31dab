// Oracle driver around the reference hmat-oss library (test infrastructure only).
//
// Runs the reference's own public C API on a point cloud given as a binary file:
//   hmat_create_clustering_median + hmat_create_clustering_max_dof   (c_default_interface.cpp:35,73)
//   hmat_create_cluster_tree                                          (c_default_interface.cpp:101)
//   hmat_create_admissibility_standard                                (c_default_interface.cpp:215)
//   hmat_create_compression_aca_plus                                  (compression.hpp:137)
//   hi.create_empty_hmatrix_admissibility / set_low_rank_epsilon /
//   assemble_generic (simple_compute callback, or advanced_compute +
//   prepare for multi-strata kernels) / gemv / get_info               (c_wrapping.hpp:41-96,233-252)
// and dumps what the parity tests compare: the cluster permutation, the leaf list,
// the leaf payloads (optional), the gemv result and wall-clock timings.
//
// Usage: ref_driver <params file>   (key=value lines, see parse_params below)
//
// The kernel callbacks are evaluated in double with a fixed operation order and no
// contraction (this file is compiled without -ffast-math), so the device kernels can
// reproduce the same entries.
#include "hmat/hmat.h"
#include "hmat_cpp_interface.hpp"
#include "h_matrix.hpp"
#include "rk_matrix.hpp"
#include "full_matrix.hpp"

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

namespace {

// hmat_iostream over a byte buffer (write_data appends, read_data consumes in order).
struct StreamBuf {
  std::vector<char> bytes;
  size_t pos = 0;
  bool overrun = false;
};
void stream_write(void* buf, size_t n, void* ud) {
  StreamBuf* s = (StreamBuf*)ud;
  s->bytes.insert(s->bytes.end(), (const char*)buf, (const char*)buf + n);
}
void stream_read(void* buf, size_t n, void* ud) {
  StreamBuf* s = (StreamBuf*)ud;
  if (s->pos + n > s->bytes.size()) {
    s->overrun = true;
    memset(buf, 0, n);
    return;
  }
  memcpy(buf, s->bytes.data() + s->pos, n);
  s->pos += n;
}

struct Params {
  std::map<std::string, std::string> kv;
  std::string get(const std::string& k, const std::string& d = "") const {
    auto it = kv.find(k);
    return it == kv.end() ? d : it->second;
  }
  double num(const std::string& k, double d) const {
    auto it = kv.find(k);
    return it == kv.end() ? d : atof(it->second.c_str());
  }
};

Params parse_params(const char* path) {
  Params p;
  FILE* f = fopen(path, "r");
  if (!f) { perror(path); exit(2); }
  char line[4096];
  while (fgets(line, sizeof line, f)) {
    char* eq = strchr(line, '=');
    if (!eq) continue;
    *eq = 0;
    std::string k(line), v(eq + 1);
    while (!v.empty() && (v.back() == '\n' || v.back() == '\r' || v.back() == ' ')) v.pop_back();
    p.kv[k] = v;
  }
  fclose(f);
  return p;
}

std::vector<char> read_file(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) { perror(path.c_str()); exit(2); }
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  std::vector<char> buf(n);
  if (n && fread(buf.data(), 1, n, f) != (size_t)n) { perror("read"); exit(2); }
  fclose(f);
  return buf;
}

void write_file(const std::string& path, const void* data, size_t bytes) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) { perror(path.c_str()); exit(2); }
  if (bytes && fwrite(data, 1, bytes, f) != bytes) { perror("write"); exit(2); }
  fclose(f);
}

// Kernel context passed to the simple_compute callback.
struct KernelCtx {
  const double* pts;  // N x 3, point-major
  int kind;           // 0 laplace_reg, 1 exp_cov, 2 helmholtz_reg
  double delta;       // regularisation of 1/(4 pi (r + delta))
  double ell;         // correlation length of exp(-r/ell)
  double nugget;      // added on the diagonal (row == col) of exp_cov
  double wavenumber;  // k of exp(i k r)
};

const double kFourPi = 4.0 * M_PI;

inline double dist(const double* a, const double* b) {
  double dx = a[0] - b[0];
  double dy = a[1] - b[1];
  double dz = a[2] - b[2];
  double s = dx * dx;
  s = s + dy * dy;
  s = s + dz * dz;
  return std::sqrt(s);
}

void real_kernel(void* vctx, int row, int col, void* result) {
  const KernelCtx* c = (const KernelCtx*)vctx;
  double r = dist(c->pts + 3 * (size_t)row, c->pts + 3 * (size_t)col);
  double v;
  if (c->kind == 0) {
    v = 1.0 / (kFourPi * (r + c->delta));
  } else {
    v = std::exp(-r / c->ell);
    if (row == col) v += c->nugget;
  }
  *(double*)result = v;
}

void complex_kernel(void* vctx, int row, int col, void* result) {
  const KernelCtx* c = (const KernelCtx*)vctx;
  double r = dist(c->pts + 3 * (size_t)row, c->pts + 3 * (size_t)col);
  double s = 1.0 / (kFourPi * (r + c->delta));
  double kr = c->wavenumber * r;
  double* out = (double*)result;
  out[0] = std::cos(kr) * s;
  out[1] = std::sin(kr) * s;
}

// Multi-strata kernel through advanced_compute (hmat.h:552-583): stratum s is w_s times the
// base kernel with its own parameter (exp_cov: ell_s; laplace: delta_s; helmholtz:
// wavenumber_s); stratum -1 sums the strata in order, as the full blocks and dense-SVD
// compressions ask for (assembly.cpp:168-180, compression.cpp:745-773).
struct StrataCtx {
  KernelCtx base;
  std::vector<double> param, weight;
};

std::complex<double> strata_value(const StrataCtx* s, int row, int col, int stratum) {
  const KernelCtx* c = &s->base;
  const double r = dist(c->pts + 3 * (size_t)row, c->pts + 3 * (size_t)col);
  std::complex<double> sum(0.0, 0.0);
  const int S = (int)s->param.size();
  for (int q = 0; q < S; ++q) {
    if (stratum >= 0 && q != stratum) continue;
    const double w = s->weight[q], a = s->param[q];
    std::complex<double> v;
    if (c->kind == 0) {
      v = std::complex<double>(w * (1.0 / (kFourPi * (r + a))), 0.0);
    } else if (c->kind == 1) {
      v = std::complex<double>(w * std::exp(-r / a), 0.0);
    } else {
      const double sc = 1.0 / (kFourPi * (r + c->delta));
      const double kr = a * r;
      v = std::complex<double>(w * (std::cos(kr) * sc), w * (std::sin(kr) * sc));
    }
    sum = stratum >= 0 ? v : std::complex<double>(sum.real() + v.real(), sum.imag() + v.imag());
  }
  return sum;
}

struct StrataBlock {
  const StrataCtx* s;
  std::vector<int> rows, cols;  // client indices of the block's rows and columns
  bool complex_;
};

void strata_release(void* p) { delete (StrataBlock*)p; }

bool g_strata_complex = false;

void strata_prepare(int row_start, int row_count, int col_start, int col_count, int* row_hmat2client, int*,
                    int* col_hmat2client, int*, void* context, hmat_block_info_t* info) {
  StrataBlock* b = new StrataBlock;
  b->s = (const StrataCtx*)context;
  b->rows.assign(row_hmat2client + row_start, row_hmat2client + row_start + row_count);
  b->cols.assign(col_hmat2client + col_start, col_hmat2client + col_start + col_count);
  b->complex_ = g_strata_complex;
  info->user_data = b;
  info->release_user_data = strata_release;
  info->number_of_strata = (int)b->s->param.size();
}

void strata_compute(struct hmat_block_compute_context_t* c) {
  const StrataBlock* b = (const StrataBlock*)c->user_data;
  double* out = (double*)c->block;
  for (int j = 0; j < c->col_count; ++j)
    for (int i = 0; i < c->row_count; ++i) {
      const std::complex<double> v =
          strata_value(b->s, b->rows[c->row_start + i], b->cols[c->col_start + j], c->stratum);
      const size_t e = i + (size_t)j * c->row_count;
      if (b->complex_) {
        out[2 * e] = v.real();
        out[2 * e + 1] = v.imag();
      } else {
        out[e] = v.real();
      }
    }
}

std::vector<double> parse_list(const std::string& s) {
  std::vector<double> v;
  size_t p = 0;
  while (p < s.size()) {
    size_t q = s.find(',', p);
    if (q == std::string::npos) q = s.size();
    if (q > p) v.push_back(atof(s.substr(p, q - p).c_str()));
    p = q + 1;
  }
  return v;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct LeafRec {
  int row_off, row_size, col_off, col_size, type, rank;
};

template <typename T>
void walk(const hmat::HMatrix<T>* h, std::vector<LeafRec>& leaves, std::vector<T>& payload, bool dump) {
  if (!h) return;
  if (!h->isLeaf()) {
    for (int i = 0; i < h->nrChild(); ++i) walk(h->getChild(i), leaves, payload, dump);
    return;
  }
  LeafRec r;
  r.row_off = h->rows()->offset();
  r.row_size = h->rows()->size();
  r.col_off = h->cols()->offset();
  r.col_size = h->cols()->size();
  if (h->isRkMatrix()) {
    r.type = 1;
    r.rank = h->rank();
    if (dump && r.rank > 0) {
      const hmat::RkMatrix<T>* rk = h->rk();
      for (int j = 0; j < r.rank; ++j)
        for (int i = 0; i < r.row_size; ++i) payload.push_back(rk->a->get(i, j));
      for (int j = 0; j < r.rank; ++j)
        for (int i = 0; i < r.col_size; ++i) payload.push_back(rk->b->get(i, j));
    }
  } else {
    r.type = 0;
    r.rank = -1;
    const hmat::FullMatrix<T>* f = h->isFullMatrix() ? h->full() : nullptr;
    if (dump && f) {
      for (int j = 0; j < r.col_size; ++j)
        for (int i = 0; i < r.row_size; ++i) payload.push_back(f->data.get(i, j));
    }
    if (!f) r.rank = -2;  // full leaf without storage (empty block)
  }
  leaves.push_back(r);
}

template <typename T>
int run(const Params& p, hmat_value_t vt) {
  const int n = (int)p.num("n", 0);
  std::vector<char> pbuf = read_file(p.get("points"));
  if ((int)(pbuf.size() / (3 * sizeof(double))) != n) {
    fprintf(stderr, "points file holds %zu bytes, expected %d points\n", pbuf.size(), n);
    return 2;
  }
  std::vector<double> pts(3 * (size_t)n);
  memcpy(pts.data(), pbuf.data(), pbuf.size());
  const std::string out = p.get("out");

  hmat_settings_t settings;
  hmat_get_parameters(&settings);
  settings.compressionMinLeafSize = (int)p.num("min_leaf", 0);
  hmat_set_parameters(&settings);

  hmat_interface_t hi;
  hmat_init_default_interface(&hi, vt);

  double t0 = now_s();
  hmat_clustering_algorithm_t* median = hmat_create_clustering_median();
  hmat_clustering_algorithm_t* algo = hmat_create_clustering_max_dof(median, (int)p.num("leaf", 64));
  hmat_cluster_tree_t* ct = hmat_create_cluster_tree(pts.data(), 3, n, algo);
  // optional second tree for the columns (same points, another leaf size)
  const int leaf_cols = (int)p.num("leaf_cols", 0);
  hmat_clustering_algorithm_t* algo_c = leaf_cols > 0 ? hmat_create_clustering_max_dof(median, leaf_cols) : nullptr;
  hmat_cluster_tree_t* cct = algo_c ? hmat_create_cluster_tree(pts.data(), 3, n, algo_c) : ct;
  hmat_admissibility_t* adm = hmat_create_admissibility_standard(p.num("eta", 2.0));
  hmat_matrix_t* M = hi.create_empty_hmatrix_admissibility(ct, cct, 0, adm);
  const double eps = p.num("eps", 1e-4);
  hi.set_low_rank_epsilon(M, eps);
  double t_build = now_s() - t0;

  KernelCtx kctx;
  kctx.pts = pts.data();
  const std::string kname = p.get("kernel", "laplace");
  kctx.kind = kname == "laplace" ? 0 : (kname == "expcov" ? 1 : 2);
  kctx.delta = p.num("delta", 0.01);
  kctx.ell = p.num("ell", 0.3);
  kctx.nugget = p.num("nugget", 0.0);
  kctx.wavenumber = p.num("wavenumber", 0.0);

  hmat_assemble_context_t ctx;
  hmat_assemble_context_init(&ctx);
  ctx.compression = hmat_create_compression_aca_plus(eps);
  ctx.user_context = &kctx;
  ctx.simple_compute = (vt == HMAT_DOUBLE_COMPLEX || vt == HMAT_SIMPLE_COMPLEX) ? complex_kernel : real_kernel;
  // optional multi-strata assembly: strata_param=a0,a1,... strata_weight=w0,w1,...
  StrataCtx sctx;
  sctx.base = kctx;
  sctx.param = parse_list(p.get("strata_param"));
  sctx.weight = parse_list(p.get("strata_weight"));
  if (!sctx.param.empty()) {
    if (sctx.weight.size() != sctx.param.size()) {
      fprintf(stderr, "strata_param and strata_weight differ in length\n");
      return 2;
    }
    g_strata_complex = vt == HMAT_DOUBLE_COMPLEX || vt == HMAT_SIMPLE_COMPLEX;
    ctx.simple_compute = nullptr;
    ctx.advanced_compute = strata_compute;
    ctx.prepare = strata_prepare;
    ctx.user_context = &sctx;
  }
  ctx.lower_symmetric = 0;
  ctx.factorization = hmat_factorization_none;
  t0 = now_s();
  int rc = 0;
  const std::string data_in = p.get("read_data");
  if (!data_in.empty()) {
    // the leaves from a data stream (write_data of this library or of another one) instead of
    // an assembly: hmat_interface_t.read_data into the matrix just built
    StreamBuf sb;
    sb.bytes = read_file(data_in);
    hi.read_data(M, stream_read, &sb);
    if (sb.pos != sb.bytes.size() || sb.overrun) {
      fprintf(stderr, "read_data consumed %zu of %zu bytes%s\n", sb.pos, sb.bytes.size(),
              sb.overrun ? " and asked for more" : "");
      return 3;
    }
  } else {
    rc = hi.assemble_generic(M, &ctx);
  }
  double t_assemble = now_s() - t0;
  if (rc) {
    fprintf(stderr, "assemble_generic failed\n");
    return 3;
  }
  // optional re-truncation of every Rk leaf at a new low-rank epsilon
  // (hmat_interface_t.set_low_rank_epsilon, then .truncate)
  const double retrunc = p.num("retrunc", 0.0);
  if (retrunc > 0.0) {
    hi.set_low_rank_epsilon(M, retrunc);
    if (hi.truncate(M)) {
      fprintf(stderr, "truncate failed\n");
      return 4;
    }
  }

  // optional data stream of the assembled matrix (hmat_interface_t.write_data)
  const std::string data_out = p.get("write_data");
  if (!data_out.empty()) {
    StreamBuf sb;
    hi.write_data(M, stream_write, &sb);
    write_file(data_out, sb.bytes.data(), sb.bytes.size());
  }

  // Cluster permutation (internal -> client).
  const int* perm = hmat_cluster_get_indices(ct);
  write_file(out + ".perm", perm, sizeof(int) * (size_t)n);
  write_file(out + ".permc", hmat_cluster_get_indices(cct), sizeof(int) * (size_t)n);

  // Leaves.
  hmat::HMatInterface<T>* hm = (hmat::HMatInterface<T>*)M;
  std::vector<LeafRec> leaves;
  std::vector<T> payload;
  const bool dump = p.num("dump_factors", 0) != 0;
  walk<T>(hm->engine().hmat, leaves, payload, dump);
  write_file(out + ".leaves", leaves.data(), leaves.size() * sizeof(LeafRec));
  if (dump) write_file(out + ".payload", payload.data(), payload.size() * sizeof(T));

  hmat_info_t info;
  memset(&info, 0, sizeof info);
  hi.get_info(M, &info);

  // gemv in client numbering, alpha = 1, beta = 0.
  const int nrhs = (int)p.num("nrhs", 1);
  const std::string trans = p.get("trans", "N");
  const int reps = (int)p.num("gemv_reps", 1);
  const int warm = (int)p.num("gemv_warmup", 0);
  double t_gemv_first = 0, t_gemv_mean = 0;
  if (!p.get("x").empty()) {
    std::vector<char> xb = read_file(p.get("x"));
    if (xb.size() != sizeof(T) * (size_t)n * nrhs) {
      fprintf(stderr, "x file holds %zu bytes, expected %zu\n", xb.size(), sizeof(T) * (size_t)n * nrhs);
      return 2;
    }
    std::vector<T> x((size_t)n * nrhs), y((size_t)n * nrhs);
    T alpha = T(1), beta = T(0);
    // the first call is timed on its own, then `warm` untimed calls, then `reps` timed ones
    for (int rep = 0; rep <= warm + reps; ++rep) {
      memcpy(x.data(), xb.data(), xb.size());
      std::fill(y.begin(), y.end(), T(0));
      t0 = now_s();
      rc = hi.gemv(trans[0], &alpha, M, x.data(), &beta, y.data(), nrhs);
      double dt = now_s() - t0;
      if (rc) { fprintf(stderr, "gemv failed\n"); return 4; }
      if (rep == 0) t_gemv_first = dt;
      else if (rep > warm) t_gemv_mean += dt / reps;
    }
    write_file(out + ".y", y.data(), y.size() * sizeof(T));
  }

  FILE* js = fopen((out + ".json").c_str(), "w");
  fprintf(js,
          "{\"n\": %d, \"leaves\": %zu, \"t_build\": %.9g, \"t_assemble\": %.9g, \"t_gemv_first\": %.9g, "
          "\"t_gemv_mean\": %.9g, \"gemv_reps\": %d, \"nrhs\": %d, \"full_count\": %zu, \"rk_count\": %zu, "
          "\"full_size\": %zu, \"rk_size\": %zu, \"compressed_size\": %zu, \"uncompressed_size\": %zu, "
          "\"nr_block_clusters\": %d, \"largest_rk_dim_rows\": %d, \"largest_rk_dim_cols\": %d, "
          "\"largest_rk_mem_rows\": %d, \"largest_rk_mem_cols\": %d, \"largest_rk_mem_rank\": %d}\n",
          n, leaves.size(), t_build, t_assemble, t_gemv_first, t_gemv_mean, reps, nrhs, info.full_count,
          info.rk_count, info.full_size, info.rk_size, info.compressed_size, info.uncompressed_size,
          info.nr_block_clusters, info.largest_rk_dim_rows, info.largest_rk_dim_cols, info.largest_rk_mem_rows,
          info.largest_rk_mem_cols, info.largest_rk_mem_rank);
  fclose(js);

  hi.destroy(M);
  hmat_delete_cluster_tree(ct);
  if (cct != ct) hmat_delete_cluster_tree(cct);
  if (algo_c) hmat_delete_clustering(algo_c);
  hmat_delete_admissibility(adm);
  hmat_delete_compression(ctx.compression);
  hmat_delete_clustering(algo);
  hmat_delete_clustering(median);
  hi.finalize();
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 2) {
    fprintf(stderr, "usage: %s <params file>\n", argv[0]);
    return 2;
  }
  Params p = parse_params(argv[1]);
  const std::string s = p.get("scalar", "D");
  if (s == "D") return run<hmat::D_t>(p, HMAT_DOUBLE_PRECISION);
  if (s == "S") return run<hmat::S_t>(p, HMAT_SIMPLE_PRECISION);
  if (s == "Z") return run<hmat::Z_t>(p, HMAT_DOUBLE_COMPLEX);
  if (s == "C") return run<hmat::C_t>(p, HMAT_SIMPLE_COMPLEX);
  fprintf(stderr, "unknown scalar type %s\n", s.c_str());
  return 2;
}
