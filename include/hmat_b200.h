/*
 * hmat_b200.h -- C ABI of the B200 engine for hmat-oss's leaf-level path.
 *
 * The engine is a drop-in for the reference's `hmat_init_default_interface` path: the
 * library exports the same C entry points (same names, same argument meaning, 0 on
 * success and non-zero on failure), and `hmat_interface_t` has the reference's field
 * order so that a program compiled against either header calls the same slots.  Linking
 * libhmat_b200.so in place of libhmat.so selects the engine.
 *
 * What runs on the GPU: dense assembly of full leaves, ACA+ (partial-ACA for very tall
 * blocks) of admissible leaves, Rk truncation, and the H-matrix-vector product
 * ('N', 'T', 'C', any number of right-hand sides).  What stays on the host: median
 * clustering, bounding boxes, the Hackbusch admissibility test and the block tree, all
 * with the reference's arithmetic so the partitions match bit for bit.
 *
 * Precision: HMAT_DOUBLE_PRECISION / HMAT_DOUBLE_COMPLEX run everything in FP64.
 * HMAT_SIMPLE_PRECISION / HMAT_SIMPLE_COMPLEX run assembly, ACA and gemv in FP32 and
 * keep FP64 for the ACA stopping-norm estimate and the QR/SVD of the truncation.
 *
 * Table slots outside this path (factorizations, solves, H-matrix products, copies,
 * serialisation, ...) are filled with functions that print an error and return a
 * failure value (non-zero, or NULL for constructors), which is how the reference's C
 * layer reports an unsupported operation.
 *
 * Interaction functions: the device cannot call host callbacks, so `simple_compute`,
 * `block_compute` and `advanced_compute` are rejected by assemble_generic (it returns 1).
 * Put a descriptor made by hmat_b200_create_assembly() in the context's `assembly` field
 * instead (the reference's "Assembly object" scenario, hmat.h:526-536).
 */
#ifndef HMAT_B200_H
#define HMAT_B200_H

#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- value types and enums (reference: include/hmat/hmat.h:57-107) ---- */
typedef enum {
  HMAT_SIMPLE_PRECISION = 0,
  HMAT_DOUBLE_PRECISION = 1,
  HMAT_SIMPLE_COMPLEX = 2,
  HMAT_DOUBLE_COMPLEX = 3
} hmat_value_t;

typedef enum {
  hmat_compress_svd,
  hmat_compress_aca_full,
  hmat_compress_aca_partial,
  hmat_compress_aca_plus,
  hmat_compress_aca_random,
  hmat_compress_rrqr
} hmat_compress_t;

typedef enum { DEFAULT_COMPRESSOR = 0, ZFP_COMPRESSOR = 1, SZ_COMPRESSOR = 2, SZ3_COMPRESSOR = 3 } hmat_FPcompress_t;

typedef enum { hmat_block_full, hmat_block_null, hmat_block_sparse } hmat_block_t;

typedef enum {
  hmat_factorization_none = -1,
  hmat_factorization_lu,
  hmat_factorization_ldlt,
  hmat_factorization_llt,
  hmat_factorization_hodlr,
  hmat_factorization_hodlrsym
} hmat_factorization_t;

/* ---- user callback types (reference: hmat.h:118-200); accepted in the context for
 *      layout compatibility, rejected at assembly time ---- */
typedef struct hmat_block_info_struct {
  hmat_block_t block_type;
  void* user_data;
  void (*release_user_data)(void* user_data);
  char (*is_guaranteed_null_row)(const struct hmat_block_info_struct* block_info, int block_row_offset, int stratum);
  char (*is_guaranteed_null_col)(const struct hmat_block_info_struct* block_info, int block_col_offset, int stratum);
  size_t needed_memory;
  int number_of_strata;
} hmat_block_info_t;

typedef struct hmat_fp_settings_struct {
  hmat_FPcompress_t compressor;
  int nb_blocs;
  float epsilonFP;
  bool compressFull;
  bool compressRk;
} hmat_fp_settings_t;

typedef void (*hmat_prepare_func_t)(int row_start, int row_count, int col_start, int col_count, int* row_hmat2client,
                                    int* row_client2hmat, int* col_hmat2client, int* col_client2hmat, void* context,
                                    hmat_block_info_t* block_info);
typedef void (*hmat_compute_func_t)(void* v_data, int block_row_start, int block_row_count, int block_col_start,
                                    int block_col_count, void* block);
typedef void (*hmat_interaction_func_t)(void* user_context, int row, int col, void* result);

/* ---- clustering (reference: hmat.h:206-330; c_default_interface.cpp:35-193) ---- */
typedef struct hmat_clustering_algorithm hmat_clustering_algorithm_t;
typedef struct hmat_cluster_tree_struct hmat_cluster_tree_t;

/* Median bisection (MedianBisectionAlgorithm, clustering.cpp:257-301). */
hmat_clustering_algorithm_t* hmat_create_clustering_median(void);
/* Copy of `algo` with at most `max_dof` points per leaf (c_default_interface.cpp:73-78). */
hmat_clustering_algorithm_t* hmat_create_clustering_max_dof(const hmat_clustering_algorithm_t* algo, int max_dof);
void hmat_delete_clustering(hmat_clustering_algorithm_t* algo);
/* Only divider 2 (bisection) is supported; other values make tree creation fail. */
void hmat_set_clustering_divider(hmat_clustering_algorithm_t* algo, int divider);
/* Cluster tree over `size` points given point-major in `coord` (c_default_interface.cpp:101-115).
 * Only dimension 3 is supported. Returns NULL on error. */
hmat_cluster_tree_t* hmat_create_cluster_tree(double* coord, int dimension, int size, hmat_clustering_algorithm_t* algo);
void hmat_delete_cluster_tree(const hmat_cluster_tree_t* tree);
int hmat_tree_nodes_count(const hmat_cluster_tree_t* tree);

typedef struct {
  int spatial_dimension;
  int dimension;
  size_t nr_tree_nodes;
} hmat_cluster_info_t;
int hmat_cluster_get_info(hmat_cluster_tree_t* tree, hmat_cluster_info_t* info);
/* internal -> client permutation of the tree (c_default_interface.cpp:191-193) */
const int* hmat_cluster_get_indices(const hmat_cluster_tree_t* tree);

/* ---- admissibility (reference: hmat.h:332-372; c_default_interface.cpp:195-240) ---- */
typedef struct {
  double eta;
  double ratio;
  size_t max_width;
  double scale;
} hmat_admissibility_param_t;
typedef struct hmat_admissibility_condition hmat_admissibility_t;
void hmat_init_admissibility_param(hmat_admissibility_param_t* p);
hmat_admissibility_t* hmat_create_admissibility(hmat_admissibility_param_t* p);
void hmat_update_admissibility(hmat_admissibility_t* cond, hmat_admissibility_param_t* p);
/* Hackbusch condition min(diam) <= eta * dist (admissibility.cpp:109-117). */
hmat_admissibility_t* hmat_create_admissibility_standard(double eta);
void hmat_delete_admissibility(hmat_admissibility_t* cond);

/* ---- compression (reference: hmat.h:376-394) ---- */
typedef struct hmat_compression_algorithm_struct hmat_compression_algorithm_t;
/* ACA+ with partial-ACA delegate (compression.hpp:134-148). */
hmat_compression_algorithm_t* hmat_create_compression_aca_plus(double epsilon);
/* Partial ACA (compression.cpp:382-533). */
hmat_compression_algorithm_t* hmat_create_compression_aca_partial(double epsilon);
/* Dense SVD, ACA-full, ACA-random and RRQR: objects are created, assembly with them fails. */
hmat_compression_algorithm_t* hmat_create_compression_svd(double epsilon);
hmat_compression_algorithm_t* hmat_create_compression_aca_full(double epsilon);
hmat_compression_algorithm_t* hmat_create_compression_aca_random(double epsilon);
hmat_compression_algorithm_t* hmat_create_compression_rrqr(double epsilon);
void hmat_delete_compression(const hmat_compression_algorithm_t* algo);

/* ---- info / settings (reference: hmat.h:404-470, 1107-1142) ---- */
typedef struct {
  int full_zeros;
  size_t full_size;
  size_t rk_size;
  size_t full_count;
  size_t rk_count;
  size_t compressed_size;
  size_t uncompressed_size;
  int nr_block_clusters;
  int largest_rk_dim_rows;
  int largest_rk_dim_cols;
  int largest_rk_mem_rows;
  int largest_rk_mem_cols;
  int largest_rk_mem_rank;
} hmat_info_t;

typedef struct {
  int wip;
} hmat_profile_t;

typedef struct hmat_matrix_struct hmat_matrix_t;

typedef struct hmat_progress_struct {
  int max;
  int current;
  void (*update)(struct hmat_progress_struct* context);
  void* user_data;
} hmat_progress_t;
hmat_progress_t* hmat_default_progress(void);

typedef struct {
  double rkRatio;
  size_t size_Rk;
  size_t size_Rk_compressed;
  double fullRatio;
  size_t size_Full;
  size_t size_Full_compressed;
  double ratio;
} hmat_FPCompressionRatio_t;

typedef void (*hmat_iostream)(void* buffer, size_t n, void* user_data);

struct hmat_block_compute_context_t {
  void* user_data;
  int row_start, row_count, col_start, col_count;
  int stratum;
  void* block;
};

/* Assembly context (reference: hmat.h:516-622).  Exactly one of `assembly`,
 * `simple_compute`, `block_compute`, `advanced_compute` is set; this engine accepts
 * only `assembly` = a descriptor from hmat_b200_create_assembly(). */
typedef struct {
  void* assembly;
  hmat_interaction_func_t simple_compute;
  hmat_compute_func_t block_compute;
  void (*advanced_compute)(struct hmat_block_compute_context_t*);
  void* user_context;
  hmat_prepare_func_t prepare;
  const hmat_compression_algorithm_t* compression;
  int lower_symmetric;
  hmat_factorization_t factorization;
  hmat_progress_t* progress;
} hmat_assemble_context_t;
void hmat_assemble_context_init(hmat_assemble_context_t* context);

typedef struct {
  hmat_factorization_t factorization;
  hmat_progress_t* progress;
} hmat_factorization_context_t;
void hmat_factorization_context_init(hmat_factorization_context_t* context);

struct hmat_get_values_context_t {
  hmat_matrix_t* matrix;
  void* values;
  int row_offset, col_offset;
  int row_size, col_size;
  int *row_indices, *col_indices;
  int renumber_rows : 1;
};

struct hmat_solve_context_t {
  void* values;
  int nr_rhs;
  int no_permutation;
  int lower;
  int upper;
  hmat_progress_t* progress;
};
void hmat_solve_context_init(struct hmat_solve_context_t* context);

typedef struct {
  hmat_value_t value_type;
  void* internal;
} hmat_procedure_t;
typedef struct {
  hmat_value_t value_type;
  const void* internal;
} hmat_leaf_procedure_t;

/* Function table (reference: hmat.h:717-1103), same slot order. */
typedef struct {
  hmat_matrix_t* (*create_empty_hmatrix_admissibility)(const hmat_cluster_tree_t* rows_tree,
                                                       const hmat_cluster_tree_t* cols_tree, int lower_symmetric,
                                                       hmat_admissibility_t* cond);
  void (*own_cluster_trees)(hmat_matrix_t* hmatrix, int owns_row, int owns_col);
  void (*set_low_rank_epsilon)(hmat_matrix_t* hmatrix, double epsilon);
  int (*assemble_generic)(hmat_matrix_t* matrix, hmat_assemble_context_t* context);
  hmat_matrix_t* (*copy)(hmat_matrix_t* hmatrix);
  hmat_matrix_t* (*copy_struct)(hmat_matrix_t* hmatrix);
  double (*norm)(hmat_matrix_t* hmatrix);
  int (*logdet)(hmat_matrix_t* hmatrix, double* result);
  int (*inverse)(hmat_matrix_t* hmatrix);
  int (*factorize_generic)(hmat_matrix_t* matrix, hmat_factorization_context_t* context);
  int (*destroy)(hmat_matrix_t* hmatrix);
  hmat_matrix_t* (*get_child)(hmat_matrix_t* hmatrix, int i, int j);
  int (*destroy_child)(hmat_matrix_t* hmatrix);
  int (*solve_generic)(hmat_matrix_t* matrix, const struct hmat_solve_context_t* context);
  int (*solve_mat)(hmat_matrix_t* hmatrix, hmat_matrix_t* hmatrixB);
  int (*solve_systems)(hmat_matrix_t* hmatrix, void* b, int nrhs);
  int (*solve_dense)(hmat_matrix_t* hmatrix, void* b, int nrhs);
  int (*transpose)(hmat_matrix_t* hmatrix);
  int (*scale)(void* alpha, hmat_matrix_t* hmatrix);
  int (*truncate)(hmat_matrix_t* hmatrix);
  int (*vector_reorder)(void* vec_b, const hmat_cluster_tree_t* rows_ct, int rows, const hmat_cluster_tree_t* cols_ct,
                        int cols);
  int (*vector_restore)(void* vec_b, const hmat_cluster_tree_t* rows_ct, int rows, const hmat_cluster_tree_t* cols_ct,
                        int cols);
  int (*gemm)(char trans_a, char trans_b, const void* alpha, hmat_matrix_t* hmatrix, hmat_matrix_t* hmatrix_b,
              const void* beta, hmat_matrix_t* hmatrix_c);
  int (*axpy)(void* a, hmat_matrix_t* x, hmat_matrix_t* hmatrix_y);
  int (*trsm)(char side, char uplo, char transa, char diag, int m, int n, void* alpha, hmat_matrix_t* A,
              int is_b_hmat, void* B);
  /* y <- alpha op(H) x + beta y, x and y column-major in client numbering, nrhs columns
   * (reference c_wrapping.hpp:233-252).  x and y are host memory. */
  int (*gemv)(char trans_a, void* alpha, hmat_matrix_t* hmatrix, void* vec_b, void* beta, void* vec_c, int nrhs);
  int (*gemm_scalar)(char trans_a, void* alpha, hmat_matrix_t* hmatrix, void* vec_b, void* beta, void* vec_c,
                     int nrhs);
  int (*full_gemm)(char trans_a, char trans_b, int mc, int nc, void* c, void* alpha, void* a, hmat_matrix_t* hmat_b,
                   void* beta);
  int (*gemm_dense)(char trans_b, char trans_x, char side, const void* alpha, hmat_matrix_t* holder, void* vec_x,
                    const void* beta, void* vec_y, int nrhs);
  int (*add_identity)(hmat_matrix_t* hmatrix, void* alpha);
  int (*init)(void);
  int (*finalize)(void);
  int (*get_info)(hmat_matrix_t* hmatrix, hmat_info_t* info);
  int (*get_profile)(hmat_matrix_t* hmatrix, hmat_profile_t* profile);
  int (*get_ratio)(hmat_matrix_t* hmatrix, hmat_FPCompressionRatio_t* ratio);
  int (*FPcompress)(hmat_matrix_t* hmatrix);
  int (*FPdecompress)(hmat_matrix_t* hmatrix);
  hmat_fp_settings_t (*GetFPCompressionSettings)(hmat_matrix_t* hmatrix);
  int (*SetFPCompressionSettings)(hmat_matrix_t* hmatrix, hmat_fp_settings_t settings);
  int (*SetFPCompressionSettingsParams)(hmat_matrix_t* hmatrix, float epsilonFP, int nb_blocs,
                                        hmat_FPcompress_t compressor, bool compressFull, bool compressRk);
  int (*dump_info)(hmat_matrix_t* hmatrix, char* prefix);
  int (*get_cluster_trees)(hmat_matrix_t* hmatrix, const hmat_cluster_tree_t** rows, const hmat_cluster_tree_t** cols);
  int (*set_cluster_trees)(hmat_matrix_t* hmatrix, const hmat_cluster_tree_t* rows, const hmat_cluster_tree_t* cols);
  int (*extract_diagonal)(hmat_matrix_t* holder, void* diag, int size);
  int (*solve_lower_triangular)(hmat_matrix_t* hmatrix, int transpose, void* b, int nrhs);
  int (*solve_lower_triangular_dense)(hmat_matrix_t* hmatrix, int transpose, void* b, int nrhs);
  int (*get_block)(struct hmat_get_values_context_t* ctx);
  int (*get_values)(struct hmat_get_values_context_t* ctx);
  int (*walk)(hmat_matrix_t* hmatrix, hmat_procedure_t* proc);
  int (*apply_on_leaf)(hmat_matrix_t* hmatrix, const hmat_leaf_procedure_t* proc);
  hmat_value_t value_type;
  void* internal;
  hmat_matrix_t* (*read_struct)(hmat_iostream readfunc, void* user_data);
  void (*write_struct)(hmat_matrix_t* matrix, hmat_iostream writefunc, void* user_data);
  void (*read_data)(hmat_matrix_t* matrix, hmat_iostream readfunc, void* user_data);
  void (*write_data)(hmat_matrix_t* matrix, hmat_iostream writefunc, void* user_data);
  void (*set_progressbar)(hmat_matrix_t* matrix, hmat_progress_t* progress);
  int (*extract_diagonal_block)(hmat_matrix_t* holder, int components, void* diag);
} hmat_interface_t;

/* Fills the table for one value type (reference: c_default_interface.cpp:242-252). */
void hmat_init_default_interface(hmat_interface_t* i, hmat_value_t type);

typedef struct {
  int compressionMinLeafSize;
  double coarseningEpsilon;
  int maxLeafSize;
  int coarsening;
  int validateNullRowCol;
  int validateCompression;
  int validateRecompression;
  int dumpTrace;
  int validationReRun;
  int validationDump;
  double validationErrorThreshold;
} hmat_settings_t;
/* Global settings (reference: c_default_interface.cpp:254-288).  Of these the engine
 * uses maxLeafSize (default leaf size of clustering algorithms without max_dof) and
 * compressionMinLeafSize: admissible blocks with max(rows, cols) below it are compressed
 * by a dense SVD, as AssemblyFunction::assemble does (assembly.cpp:59-64). */
void hmat_get_parameters(hmat_settings_t* settings);
int hmat_set_parameters(hmat_settings_t* settings);
const char* hmat_get_version(void);

/* ======================================================================================
 * B200 extensions (no counterpart in the reference's C API).
 * ====================================================================================== */

/* Interaction kernels evaluated on the device:
 *   HMAT_B200_LAPLACE_REG    K = 1 / (4 pi (r + delta))
 *   HMAT_B200_EXP_COV        K = exp(-r / ell) + nugget * [row == col]
 *   HMAT_B200_HELMHOLTZ_REG  K = exp(i k r) / (4 pi (r + delta))   (complex types only) */
typedef enum { HMAT_B200_LAPLACE_REG = 0, HMAT_B200_EXP_COV = 1, HMAT_B200_HELMHOLTZ_REG = 2 } hmat_b200_kernel_kind_t;

typedef struct {
  hmat_b200_kernel_kind_t kind;
  double delta;
  double ell;
  double nugget;
  double wavenumber;
} hmat_b200_kernel_t;

/* Assembly descriptor for hmat_assemble_context_t.assembly: kernel + the points it is
 * evaluated on (client numbering, point-major xyz, copied).  NULL on bad input. */
void* hmat_b200_create_assembly(const hmat_b200_kernel_t* kernel, const double* coord, int n_points);
/* Assembly descriptor of a multi-strata kernel: the sum of `nstrata` (1 to 8) strata, stratum q
 * being weight[q] times `kernel` with its parameter replaced by param[q] (the correlation length
 * of the exponential covariance, without the nugget; the regularisation delta of the Laplace
 * kernel; the wavenumber of the Helmholtz kernel, whose amplitude keeps kernel->delta).  It
 * replaces the reference's advanced_compute callback with prepare() setting number_of_strata
 * (hmat.h:552-583): admissible blocks compressed by ACA+ or partial ACA are compressed stratum
 * by stratum, each further stratum added to the truncated sum as compress() does
 * (compression.cpp:745-773, RkMatrix::formattedAddParts rk_matrix.cpp:846-1009); full blocks
 * and the dense-SVD compression of small blocks take the sum.  NULL on bad input. */
void* hmat_b200_create_assembly_strata(const hmat_b200_kernel_t* kernel, const double* coord, int n_points,
                                       int nstrata, const double* param, const double* weight);
void hmat_b200_delete_assembly(void* assembly);

/* gemv on device buffers (x, y column-major, client numbering, leading dimension = the
 * vector length), enqueued on `stream` (a cudaStream_t, NULL for the engine's own) and
 * not synchronised.  Same maths and return convention as hmat_interface_t.gemv (reference:
 * c_wrapping.hpp:233-252, with the buffers on the device).  The device that was current when
 * the matrix was assembled must be current (otherwise the call fails).  The return code
 * covers the arguments and the launches only: a kernel whose bounded wait for a bulk copy
 * gives up marks the matrix's status flag and leaves y invalid; read it with
 * hmat_b200_gemv_status once the product is complete. */
int hmat_b200_gemv_device(hmat_matrix_t* hmatrix, char trans, const void* alpha, const void* x_dev,
                          const void* beta, void* y_dev, int nrhs, void* stream);

/* Status of the device products of `hmatrix` (hmat_b200_gemv_device, _noalloc, and the
 * leaf gradients): synchronises `stream` (NULL: the matrix's own stream), then sets *failed
 * to 1 if one of them stopped since the last query because a kernel's wait for a bulk copy
 * gave up, 2 if a unit of the product's schedule failed the kernels' own checks of its copies
 * (sizes, alignment, stage bounds) and was skipped (in both cases the results are not valid),
 * else 0, and clears the flag.  Allocates nothing.
 * The C table's gemv checks the same flag itself and returns 1.  Returns 0, or non-zero
 * on a bad argument.  No counterpart in the reference (its products run on the host). */
int hmat_b200_gemv_status(hmat_matrix_t* hmatrix, void* stream, int* failed);

/* hmat_b200_gemv_device for callers that cannot allocate device memory when they
 * multiply (no counterpart in the reference's C API).  Callers inside a caching
 * allocator or memory pool they do not control, inside callbacks where cudaMalloc /
 * cudaFree would synchronise or deadlock, or in loops that forbid allocation after
 * start-up can use it: it calls no cudaMalloc, cudaFree or other allocating routine.
 * Its scratch (x in cluster order and the per-leaf B^T x values) is
 * one fixed 16 MiB device array compiled into the library: every GPU on which the
 * library's device code is loaded holds it until the process exits.  Matrices whose
 * product needs more scratch than that are rejected with a non-zero return and an
 * error message (use hmat_b200_gemv_device for them).  The first call on each device
 * looks up the array's device address (with that device current); make that first call
 * before any stream capture.  Every call shares the one array, so calls that can overlap
 * on the GPU (different streams, or different host threads, without ordering between
 * them) race: order them on one stream.  The array keeps the previous call's contents;
 * nothing in it needs to start at zero, since each product overwrites what it reads.
 * The address is looked up once per process and device; a cudaDeviceReset is not supported.
 * Same arguments, maths and return convention as hmat_b200_gemv_device (the matrix's device
 * current; a bulk-copy wait that gives up is reported by hmat_b200_gemv_status, through a
 * flag allocated with the matrix, not in the shared array); `stream` NULL means the
 * matrix's own stream. */
int hmat_b200_gemv_device_noalloc(hmat_matrix_t* hmatrix, char trans, const void* alpha, const void* x_dev,
                                  const void* beta, void* y_dev, int nrhs, void* stream);

/* Batches of independent H-matrices (no counterpart in the reference, whose
 * assemble_generic and gemv take one matrix, c_wrapping.hpp:57-96 and 233-252).
 * hmat_b200_batch_create combines `count` matrices made by create_empty_hmatrix_admissibility
 * (each on one cluster tree for rows and columns, one value type and one low-rank epsilon; they
 * are not assembled and stay owned by the caller) into one block-diagonal matrix: their
 * cluster trees side by side, member i's rows and columns numbered from row_base[i], its leaves
 * from leaf_base[i] (hmat_b200_batch_offsets, count + 1 entries each).  The batch is an
 * ordinary matrix for every other entry point (gemv, hmat_b200_gemv_device, the leaf table and
 * payloads, get_info, destroy through the table), so all members are assembled and multiplied
 * by one launch per phase; vectors are the members' vectors stacked (column-major, N_total x
 * nrhs).  Each member's leaves and ranks are those of its own assembly.  It owns the combined
 * cluster tree; NULL on error.
 * hmat_b200_batch_assemble assembles every member with its own descriptor from
 * hmat_b200_create_assembly (assemblies[i] on member i's points; one kernel kind and nugget,
 * each member its own correlation length, regularisation or wavenumber) and one compression
 * algorithm (ACA+ or partial ACA). */
hmat_matrix_t* hmat_b200_batch_create(hmat_matrix_t* const* matrices, int count);
int hmat_b200_batch_offsets(hmat_matrix_t* batch, int* row_base, int* leaf_base);
int hmat_b200_batch_assemble(hmat_matrix_t* batch, void* const* assemblies,
                             const hmat_compression_algorithm_t* compression);

/* Leaf table: `n` leaves in the reference's depth-first order, 6 ints each: row offset,
 * rows, col offset, cols (cluster numbering), type (0 full, 1 rk), rank (-1 for full). */
int hmat_b200_leaf_count(hmat_matrix_t* hmatrix);
int hmat_b200_leaf_table(hmat_matrix_t* hmatrix, int* out);
/* Payload of leaf `leaf` copied to host memory `out` (full: m x n column-major; rk: A
 * (m x k) then B (n x k)); returns the number of scalars, or -1. */
long long hmat_b200_leaf_payload(hmat_matrix_t* hmatrix, int leaf, void* out);

/* Canonical payload layout of the assembled leaves: leaves in leaf-table order, each full
 * leaf as F (m x n), each Rk leaf as A (m x k) then B (n x k), column-major, rank-0 leaves
 * empty.  offsets[leaf] (leaf_count entries, may be NULL) and the total number of scalars.
 * (The device storage itself is internal: row panels and B transposed.) */
int hmat_b200_payload_layout(hmat_matrix_t* hmatrix, long long* offsets, long long* total);

/* Leaf-factor gradients of y = H x for an output gradient `r` (device buffers, client
 * numbering, 1 to 16 columns), written into `grad` (device, canonical payload layout),
 * added to its contents when `accumulate` is non-zero:
 *   dF = r_I x_J^T                                         per full leaf F
 *   dA = r_I (B^T x_J)^T,  dB = x_J (A^T r_I)^T             per Rk leaf A B^T
 * The gradient with respect to x is gemv('T') of r.  Real value types only. */
int hmat_b200_leaf_gradients(hmat_matrix_t* hmatrix, const void* x_dev, const void* r_dev, int nrhs, void* grad,
                             int accumulate, void* stream);

/* The whole backward pass of y = H x at the output gradient r (device buffers, client
 * numbering, 1 to 16 columns): dx = H^T r into dx_dev, and the leaf gradients of
 * hmat_b200_leaf_gradients into grad (added when `accumulate`).  One pass: the transposed
 * product's A^T r serves as the gradients' w, so it costs one transposed product plus the
 * gradient kernels and one B^T x.  Real value types only.  No counterpart in the reference
 * (its transposed product is RkMatrix::gemv 'T', rk_matrix.cpp:156-206). */
int hmat_b200_gemv_adjoint(hmat_matrix_t* hmatrix, const void* x_dev, const void* r_dev, int nrhs, void* dx_dev,
                           void* grad, int accumulate, void* stream);

/* One eager product y = op(H) x on device buffers (1 to 16 right-hand sides), timed per
 * phase with CUDA events: ms3 = device ms of [gather, z-phase, y-phase], bytes3 = their
 * algorithmic bytes (x read and x_rm written; the B (A for 'T') factors; full leaves,
 * A (B) factors and the y write).  Synchronous. */
int hmat_b200_gemv_profile(hmat_matrix_t* hmatrix, char trans, const void* x_dev, void* y_dev, int nrhs, double* ms3,
                           double* bytes3);

/* Number of kernel launches one product with nrhs right-hand sides makes (gather, the
 * z-phase launches, z-reduce, y-phase, final pass; per tile of right-hand sides), or -1
 * (with hmat_b200_last_error set) on error.  No counterpart in the reference. */
int hmat_b200_gemv_launches(hmat_matrix_t* hmatrix, char trans, int nrhs);

/* Device time of the last phases on this matrix, milliseconds: [0] full leaves and the
 * placement of the compressed leaves in the product's layout, [1] ACA, [2] truncation (+
 * compaction), [3] last gemv. */
int hmat_b200_phase_times(hmat_matrix_t* hmatrix, double* out4);

/* ACA autotuner report of the last assembly, per leaf-size bucket b (0: m, n <= 64; 1: m + n
 * below 2,048; 2: below 8,192; 3: above): shape4[b] = CTA size of the ACA kernel that ran the
 * bucket (0 = a warp per leaf, 64, 128, 256 or 512; -1 = no leaf), tuned4[b] = 0 (default
 * shape or HMAT_B200_ACA_SHAPE), 1 (measured during that assembly), 2 (measured by an earlier
 * assembly of the process), rate20[5 b + s] = leaf cost ((m + n) min(m, n)) per ms that shape
 * s (warp, 64, 128, 256, 512) reached on its sample, 0 when not run.  No counterpart in the
 * reference. */
int hmat_b200_aca_shapes(hmat_matrix_t* hmatrix, int* shape4, int* tuned4, double* rate20);

/* The gemv tuner's choice for the matrix's 'N' product schedule (no counterpart in the
 * reference): choice2[0] = units per chunk of long z tasks (8, 16 or 32), choice2[1] = y-phase
 * unit width (0 the widest that fits a pipeline stage, 1 half of it); *how = 0 default, 1
 * measured on this matrix, 2 taken from an earlier measurement of the process; ms5 = device ms
 * of the z-phase with chunks of 8, 16 and 32 units, and of the y-phase with the widest and the
 * half-width units (0 where not measured).  0, or non-zero before assembly. */
int hmat_b200_gemv_tuning(hmat_matrix_t* hmatrix, int* choice2, int* how, double* ms5);

/* Last error message of the calling thread ("" if none). */
const char* hmat_b200_last_error(void);
/* Clears the calling thread's last error (for the table entries that return no status,
 * such as write_struct / read_data: clear, call, then read hmat_b200_last_error). */
void hmat_b200_clear_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* HMAT_B200_H */
