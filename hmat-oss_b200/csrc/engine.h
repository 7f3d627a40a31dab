// The B200 engine: device residency and phase orchestration for one H-matrix.
//
// Plays the role of the reference's IEngine<T> / DefaultEngine<T> pair
// (iengine.hpp:31-98, default_engine.cpp:94-141) for the leaf-level path: assembly and
// gemv.  The block tree is built on the host (host.h); this class flattens it into
// device-resident leaf descriptors, runs the assembly phases and keeps the gemv
// schedule and its CUDA graph.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "common.cuh"
#include "host.h"

namespace hmatb200 {

struct AssemblyDesc {
  KernelParams kp;
  std::vector<double> pts;    // client numbering, point-major
  // Optional, one per point (client numbering): the kernel's parameter for the blocks of that
  // point's rows, in place of kp's (the correlation length of the exponential covariance, the
  // regularisation of the Laplace kernels, the Helmholtz wavenumber).  Batches of independent
  // matrices with their own kernels use it: a block's rows and columns belong to one matrix.
  std::vector<double> param;
  // Optional multi-strata kernel: a_0 .. a_{S-1} then w_0 .. w_{S-1} (stratum q is w_q times
  // the kernel with its parameter set to a_q); empty for a plain kernel.
  std::vector<double> strata;
};

struct LeafGrad;

class EngineBase {
 public:
  virtual ~EngineBase() {}
  // method: 0 ACA+, 1 partial ACA.  eps_aca is the compression's epsilon, eps_trunc the
  // matrix's low-rank epsilon; admissible blocks with max(m, n) < svd_below are
  // compressed by dense SVD instead.
  virtual void assemble(const AssemblyDesc& a, int method, double eps_aca, double eps_trunc, int svd_below) = 0;
  virtual void gemv_device(char trans, const void* alpha, const void* x, const void* beta, void* y, int nrhs,
                           cudaStream_t user_stream) = 0;
  virtual void gemv_host(char trans, const void* alpha, const void* x, const void* beta, void* y, int nrhs) = 0;
  virtual long long leaf_payload(int leaf, void* out) = 0;
  // Canonical payload layout (leaf order; full: m x n, Rk: A m x k then B n x k, column-major).
  virtual void payload_layout(long long* offsets, long long* total) = 0;
  virtual void leaf_gradients(const void* x, const void* r, int nrhs, void* grad, bool accumulate,
                              cudaStream_t user_stream) = 0;
  // dx = H^T r and the leaf gradients (leaf_gradients) in one pass.
  virtual void gemv_adjoint(const void* x, const void* r, int nrhs, void* dx, void* grad, bool accumulate,
                            cudaStream_t user_stream) = 0;
  virtual void retruncate(double eps) = 0;
  // Loads stored leaves: ranks[i] (-1 for full leaves) and the canonical payload of every
  // leaf (payload_layout order, host memory); the matrix is then assembled.
  virtual void load_leaves(const int* ranks_in, const void* canonical) = 0;
  // One eager product on device buffers with events between its phases: device ms of
  // [gather, z-phase, y-phase] and their algorithmic bytes (nrhs <= 16).
  virtual void profile_gemv(char trans, const void* x, void* y, int nrhs, double* ms3, double* bytes3) = 0;
  // Bytes of scratch one eager product needs (x in cluster order + the z buffer), and that
  // product run eagerly with its scratch carved from `scratch` (no allocation, no graph).
  virtual size_t gemv_scratch_bytes() const = 0;
  // Kernel launches of one product (gather, z-phase classes, z-reduce, y-phase, final pass).
  virtual int gemv_launches(char trans, int nrhs) const = 0;
  virtual void gemv_device_with_scratch(char trans, const void* alpha, const void* x, const void* beta, void* y,
                                        int nrhs, cudaStream_t stream, void* scratch, size_t scratch_bytes) = 0;
  // 1 if a product of this matrix on the device entry points stopped because a kernel's wait
  // for a bulk copy gave up since the last query (the flag is then cleared), else 0.
  // Synchronises `stream` (NULL: the matrix's own stream).
  virtual int gemv_status(cudaStream_t stream) = 0;

  bool assembled = false;
  int device = 0;  // the CUDA device the matrix lives on (current when it was created)
  std::vector<int> ranks;  // per leaf, -1 for full leaves
  double times_ms[4] = {0, 0, 0, 0};
  // ACA autotuner report of the last assembly, per leaf-size bucket (m, n <= 64; m + n below
  // 2,048; below 8,192; above): the CTA size used (0 = warp per leaf, 64, 128, 256, 512; -1 =
  // no leaves), how it was chosen (0 default or forced, 1 measured now, 2 cached from an
  // earlier assembly of the process) and the measured leaf cost per ms of each shape (0 = not
  // run).
  // Gemv tuner report of the last plan: the chosen z chunk size (units) and y unit width (0
  // widest, 1 half), how (0 default, 1 measured now, 2 cached) and the measured device ms:
  // z-phase with chunks of 8, 16, 32 units, y-phase with widest and half-width units.
  int gemv_choice[2] = {16, 0};
  int gemv_tuned = 0;
  double gemv_rate[5] = {};
  int aca_shape[4] = {-1, -1, -1, -1};
  int aca_tuned[4] = {0, 0, 0, 0};
  double aca_rate[4][5] = {};
};

std::unique_ptr<EngineBase> make_engine(int value_type, const ClusterTree* rows, const ClusterTree* cols,
                                        const BlockTree* bt);

}  // namespace hmatb200
