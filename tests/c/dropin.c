/*
 * A C program written against the reference's own header (hmat/hmat.h of hmat-oss), linked
 * against libhmat_b200.so instead of libhmat: it shows that a caller of the reference builds
 * and runs unchanged, apart from the interaction function (a device kernel descriptor in the
 * context's `assembly` field, whose two entry points are declared below since the reference
 * header does not know them).  The flow follows the reference's examples/c-simple-cylinder.c:
 * points on a cylinder, median clustering, standard admissibility, create_empty_hmatrix_admissibility,
 * get_info, assemble_generic, gemv, destroy.
 *
 *   dropin host     host-only part: clustering, block tree, get_info before assembly, the
 *                   refusal of a host callback (simple_compute) with return code 1
 *   dropin forward  the same through the table forwarder of INTEGRATION.md (HMAT_ENGINE=b200
 *                   selects this library by dlopen inside hmat_init_default_interface)
 *   dropin gpu      assembly on the device (FP64 and the mixed FP32 engine) and gemv 'N' / 'T'
 *                   against the dense kernel product computed here in double precision
 * Exit status 0 on success.
 */
#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hmat/hmat.h"

/* ---- the B200 engine's kernel descriptor (include/hmat_b200.h of this repository) ---- */
typedef struct {
  int kind; /* 0: regularised Laplace 1 / (4 pi (r + delta)) */
  double delta, ell, nugget, wavenumber;
} b200_kernel_t;
void* hmat_b200_create_assembly(const b200_kernel_t* kernel, const double* coord, int n_points);
void hmat_b200_delete_assembly(void* assembly);

/* ---- the table forwarder a maintainer adds to hmat_init_default_interface ---- */
typedef void (*init_fn)(hmat_interface_t*, hmat_value_t);

static int forward_to_b200(hmat_interface_t* hi, hmat_value_t type) {
  const char* e = getenv("HMAT_ENGINE");
  if (!e || strcmp(e, "b200") != 0) return 0;
  void* lib = dlopen("libhmat_b200.so", RTLD_NOW | RTLD_LOCAL);
  init_fn init = lib ? (init_fn)dlsym(lib, "hmat_init_default_interface") : NULL;
  if (!init) { /* asked for by name: no silent CPU fallback */
    fprintf(stderr, "HMAT_ENGINE=b200 but libhmat_b200.so cannot be loaded: %s\n", dlerror());
    exit(1);
  }
  init(hi, type);
  return 1;
}

#define CHECK(c)                                                       \
  do {                                                                 \
    if (!(c)) {                                                        \
      fprintf(stderr, "dropin: check failed at line %d: %s\n", __LINE__, #c); \
      exit(2);                                                         \
    }                                                                  \
  } while (0)

static double* cylinder(int n_theta, int n_z) {
  double* p = malloc(sizeof(double) * 3 * n_theta * n_z);
  for (int j = 0; j < n_z; ++j)
    for (int i = 0; i < n_theta; ++i) {
      const double th = 2.0 * M_PI * i / n_theta;
      double* q = p + 3 * (j * n_theta + i);
      q[0] = cos(th);
      q[1] = sin(th);
      q[2] = 4.0 * j / (n_z - 1);
    }
  return p;
}

static void refuse_callback(void* ctx, int row, int col, void* result) {
  (void)ctx;
  (void)row;
  (void)col;
  *(double*)result = 0.0;
}

/* y = K x with the dense FP64 kernel (client numbering), and its transpose (K is symmetric). */
static void dense_product(const double* p, int n, const double* x, double* y) {
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int j = 0; j < n; ++j) {
      const double dx = p[3 * i] - p[3 * j], dy = p[3 * i + 1] - p[3 * j + 1], dz = p[3 * i + 2] - p[3 * j + 2];
      s += x[j] / (4.0 * M_PI * (sqrt(dx * dx + dy * dy + dz * dz) + 0.01));
    }
    y[i] = s;
  }
}

static double rel_err(const double* a, const double* b, int n) {
  double num = 0, den = 0;
  for (int i = 0; i < n; ++i) {
    num += (a[i] - b[i]) * (a[i] - b[i]);
    den += b[i] * b[i];
  }
  return sqrt(num / den);
}

int main(int argc, char** argv) {
  const char* mode = argc > 1 ? argv[1] : "host";
  const int n_theta = 40, n_z = 50, n = n_theta * n_z;
  double* points = cylinder(n_theta, n_z);

  hmat_interface_t hmat;
  if (!strcmp(mode, "forward")) {
    CHECK(forward_to_b200(&hmat, HMAT_DOUBLE_PRECISION));
  } else {
    hmat_init_default_interface(&hmat, HMAT_DOUBLE_PRECISION);
  }
  CHECK(hmat.value_type == HMAT_DOUBLE_PRECISION);

  hmat_settings_t settings;
  hmat_get_parameters(&settings);
  settings.compressionMinLeafSize = 0; /* ACA+ on every admissible block */
  CHECK(hmat_set_parameters(&settings) == 0);

  hmat_clustering_algorithm_t* median = hmat_create_clustering_median();
  hmat_clustering_algorithm_t* clustering = hmat_create_clustering_max_dof(median, 32);
  hmat_cluster_tree_t* cluster_tree = hmat_create_cluster_tree(points, 3, n, clustering);
  CHECK(cluster_tree != NULL);
  CHECK(hmat_tree_nodes_count(cluster_tree) > 1);
  hmat_admissibility_t* adm = hmat_create_admissibility_standard(2.0);
  hmat_matrix_t* hmatrix = hmat.create_empty_hmatrix_admissibility(cluster_tree, cluster_tree, 0, adm);
  CHECK(hmatrix != NULL);
  hmat.set_low_rank_epsilon(hmatrix, 1e-4);
  hmat_info_t info;
  CHECK(hmat.get_info(hmatrix, &info) == 0);
  CHECK(info.nr_block_clusters > 1);
  printf("HMatrix node count = %d\n", info.nr_block_clusters);

  /* a host interaction callback cannot run on the device: refused with 1 */
  hmat_assemble_context_t ctx;
  hmat_assemble_context_init(&ctx);
  ctx.simple_compute = refuse_callback;
  ctx.compression = hmat_create_compression_aca_plus(1e-4);
  CHECK(hmat.assemble_generic(hmatrix, &ctx) == 1);

  if (!strcmp(mode, "gpu")) {
    double* x = malloc(sizeof(double) * 2 * n);
    double* y = malloc(sizeof(double) * 2 * n);
    double* yd = malloc(sizeof(double) * n);
    srand(3);
    for (int i = 0; i < 2 * n; ++i) x[i] = (double)rand() / RAND_MAX - 0.5;
    dense_product(points, n, x, yd);
    for (int vt = 0; vt < 2; ++vt) {
      hmat_interface_t hi;
      hmat_init_default_interface(&hi, vt == 0 ? HMAT_DOUBLE_PRECISION : HMAT_SIMPLE_PRECISION);
      hmat_matrix_t* m = hi.create_empty_hmatrix_admissibility(cluster_tree, cluster_tree, 0, adm);
      hi.set_low_rank_epsilon(m, 1e-4);
      b200_kernel_t k = {0, 0.01, 0.0, 0.0, 0.0};
      hmat_assemble_context_t c;
      hmat_assemble_context_init(&c);
      c.assembly = hmat_b200_create_assembly(&k, points, n);
      c.compression = ctx.compression;
      CHECK(c.assembly != NULL);
      CHECK(hi.assemble_generic(m, &c) == 0);
      hmat_info_t inf;
      CHECK(hi.get_info(m, &inf) == 0);
      CHECK(inf.rk_count > 0 && inf.full_count > 0);
      for (int t = 0; t < 2; ++t) {
        const char trans = t == 0 ? 'N' : 'T';
        double err;
        if (vt == 0) {
          double alpha = 1.0, beta = 0.0;
          memcpy(y, x, sizeof(double) * 2 * n); /* gemv permutes x in place and restores it */
          double* xx = malloc(sizeof(double) * 2 * n);
          memcpy(xx, x, sizeof(double) * 2 * n);
          CHECK(hi.gemv(trans, &alpha, m, xx, &beta, y, 2) == 0);
          CHECK(memcmp(xx, x, sizeof(double) * 2 * n) == 0);
          free(xx);
          err = rel_err(y, yd, n);
        } else {
          float alpha = 1.0f, beta = 0.0f;
          float* xf = malloc(sizeof(float) * n);
          float* yf = malloc(sizeof(float) * n);
          for (int i = 0; i < n; ++i) xf[i] = (float)x[i];
          CHECK(hi.gemv(trans, &alpha, m, xf, &beta, yf, 1) == 0);
          for (int i = 0; i < n; ++i) y[i] = yf[i];
          free(xf);
          free(yf);
          err = rel_err(y, yd, n);
        }
        printf("%s gemv '%c': relative error against the dense product %.3e\n", vt == 0 ? "FP64" : "mixed",
               trans, err);
        CHECK(err < 1e-3);
      }
      hmat_b200_delete_assembly(c.assembly);
      CHECK(hi.destroy(m) == 0);
      hi.finalize();
    }
    free(x);
    free(y);
    free(yd);
  }

  hmat_delete_compression(ctx.compression);
  CHECK(hmat.destroy(hmatrix) == 0);
  hmat_delete_admissibility(adm);
  hmat_delete_cluster_tree(cluster_tree);
  hmat_delete_clustering(clustering);
  hmat_delete_clustering(median);
  hmat.finalize();
  free(points);
  printf("dropin %s ok\n", mode);
  return 0;
}
