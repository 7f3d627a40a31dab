/* hmat_oracle.h -- CPU restatement of hmat-oss's leaf-level path (TEST INFRASTRUCTURE ONLY).
 *
 * This library is the checker for the B200 engine.  Only the test suite, the smoke
 * check and the CPU-baseline leg of the benchmark load it; the product never links or
 * calls it.  Everything runs in FP64 (double / double complex), following the
 * reference's algorithms step by step:
 *   - median-bisection cluster tree        clustering.cpp:108-152,257-301,550-565
 *   - axis-aligned boxes, Hackbusch eta     cluster_tree.cpp:212-230,249,287; admissibility.cpp:38-49,95-117
 *   - block tree / leaf typing              h_matrix.cpp:144-221
 *   - dense leaf assembly                   assembly.cpp:49-91
 *   - ACA+ and its partial-ACA delegate     compression.cpp:81-220,382-533,553-724
 *   - Rk truncation (QR, QR, SVD, findK)    rk_matrix.cpp:490-585; scalar_array.cpp:97-115,927-966
 *   - H-matrix-vector product               h_matrix.cpp:792-857; rk_matrix.cpp:156-206
 * Its parity with the reference itself is pinned by tests that run the reference
 * library (built from its own sources by oracle/Makefile.ref) on the same inputs, and by
 * the golden fixtures under tests/golden/ that those runs produced.
 */
#ifndef HMAT_ORACLE_H
#define HMAT_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_hmat oracle_hmat;

/* Kernel kinds, evaluated in double with the operation order of the tests' callbacks:
 *  0: 1 / (4 pi (r + delta))                     (regularised Laplace)
 *  1: exp(-r / ell) + nugget * [row == col]      (exponential covariance)
 *  2: exp(i k r) / (4 pi (r + delta))            (regularised Helmholtz, complex) */
typedef struct {
  int kind;
  double delta, ell, nugget, wavenumber;
  /* Strata kernels (nstrata >= 1, at most 8; 0 for the plain kernel; assembly through
   * advanced_compute, hmat.h:552-583): stratum s is sweight[s] times the kernel with its
   * parameter (ell, delta or wavenumber) replaced by sparam[s], the nugget left out; full
   * leaves and dense-SVD compressions take the sum of the strata in order, and with two
   * strata or more ACA+ leaves are compressed stratum by stratum (compression.cpp:745-773). */
  int nstrata;
  double sparam[8], sweight[8];
} oracle_kernel;

/* Builds the cluster tree on n points (point-major xyz) with leaves of at most
 * `leaf_size` points, and the block tree with the standard admissibility `eta`. */
oracle_hmat* oracle_create(const double* pts, int n, int leaf_size, double eta);
/* Same with separate row and column trees (same points, different leaf sizes). */
oracle_hmat* oracle_create2(const double* pts, int n, int leaf_rows, int leaf_cols, double eta);
void oracle_destroy(oracle_hmat* h);

/* Internal -> client permutation (n ints) of the row (column) tree, as
 * hmat_cluster_get_indices returns it. */
void oracle_perm(const oracle_hmat* h, int* out);
void oracle_perm_cols(const oracle_hmat* h, int* out);
int oracle_num_leaves(const oracle_hmat* h);
/* 6 ints per leaf: row offset, row size, col offset, col size, type (0 full, 1 rk), rank
 * (-1 for full leaves).  Leaves come in the reference's depth-first order. */
void oracle_leaves(const oracle_hmat* h, int* out);
/* Number of cluster-tree nodes and their (offset, size, first child, second child). */
int oracle_num_nodes(const oracle_hmat* h);
void oracle_nodes(const oracle_hmat* h, int* out);
/* hmat_info_t fields in order: full_count, rk_count, full_size, rk_size, compressed_size,
 * uncompressed_size, nr_block_clusters, largest_rk_dim_rows, largest_rk_dim_cols,
 * largest_rk_mem_rows, largest_rk_mem_cols, largest_rk_mem_rank. */
void oracle_info(const oracle_hmat* h, long long* out);

/* Assembles every leaf: dense evaluation for full leaves, ACA+ then truncation at
 * `epsilon` for admissible ones.  is_complex selects the double complex path (kernel 2).
 * Returns 0 on success. */
int oracle_assemble(oracle_hmat* h, const oracle_kernel* k, double epsilon, int is_complex);
/* Same, compressing admissible blocks with max(m, n) < min_leaf by a dense SVD (the
 * reference's compressionMinLeafSize setting, assembly.cpp:59-64). */
int oracle_assemble2(oracle_hmat* h, const oracle_kernel* k, double epsilon, int is_complex, int min_leaf);

/* Payload size in scalars of leaf `i` (m*n for full, k*(m+n) for rk) and a copy of it:
 * full leaves column-major m x n; rk leaves A (m x k) then B (n x k), column-major.
 * Complex payloads are interleaved (re, im) pairs. */
/* Re-truncates every Rk leaf at `epsilon` (HMatrix::truncate, h_matrix.cpp:2107-2123). */
int oracle_retruncate(oracle_hmat* h, double epsilon);

long long oracle_leaf_payload_size(const oracle_hmat* h, int i);
void oracle_leaf_payload(const oracle_hmat* h, int i, double* out);

/* y = op(H) x for nrhs right-hand sides, client numbering, column-major n x nrhs.
 * trans is 'N', 'T' or (complex) 'C'. */
int oracle_gemv(const oracle_hmat* h, char trans, int nrhs, const double* x, double* y);

/* One kernel entry in client numbering (2 doubles written when complex). */
void oracle_kernel_eval(const oracle_hmat* h, const oracle_kernel* k, int row, int col, double* out);

#ifdef __cplusplus
}
#endif
#endif
