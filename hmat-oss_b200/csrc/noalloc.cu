// hmat_b200_gemv_device_noalloc: the device gemv for callers that cannot allocate.
//
// Some callers may not allocate GPU memory at the moment they need a product: code that
// runs under a memory pool or allocator it does not own (a framework's caching allocator,
// a solver that has reserved all device memory up front), code inside a callback where
// cudaMalloc / cudaFree would synchronise the device or deadlock, or hard real-time loops
// that forbid allocation after start-up.  hmat_b200_gemv_device allocates its scratch
// lazily (the cluster-ordered copy of x and the per-leaf z = B^T x values) and builds a CUDA
// graph on first use; this variant does neither.  Its scratch is one file-scope device
// array of fixed size, reserved by every GPU that loads this library's device code and
// held until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine.h"
#include "hmat_b200.h"

namespace hmatb200 {
EngineBase* existing_engine(hmat_matrix_t* m);
int report_failure(const char* where, const std::string& msg);
}  // namespace hmatb200

using namespace hmatb200;

namespace {

// 16 MiB: the cluster-ordered x (N x 16 scalars) plus the z buffer of the matrix must fit.
// The address looked up for a device stays valid for the life of the process's context on
// that device; a cudaDeviceReset (which destroys that context) is not supported.
constexpr size_t kNoAllocScratchBytes = 16u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device, looked up once per device
// (the array's host-side name is only a stand-in for the symbol, not a device address).
void* scratch_address(int device) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw Error(std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") + cudaGetErrorString(e));
    g_scratch_addr[device] = p;
  }
  return g_scratch_addr[device];
}

}  // namespace

extern "C" int hmat_b200_gemv_device_noalloc(hmat_matrix_t* m, char trans, const void* alpha, const void* x_dev,
                                             const void* beta, void* y_dev, int nrhs, void* stream) {
  try {
    if (!m || !alpha || !beta || (nrhs > 0 && (!x_dev || !y_dev))) throw Error("null argument");
    EngineBase* e = existing_engine(m);
    if (!e || !e->assembled) throw Error("matrix is not assembled");
    const size_t need = e->gemv_scratch_bytes();
    if (need > kNoAllocScratchBytes)
      throw Error("matrix needs " + std::to_string(need) + " bytes of gemv scratch, more than the " +
                  std::to_string(kNoAllocScratchBytes) + " bytes this entry point holds; use hmat_b200_gemv_device");
    // the scratch address is looked up on the matrix's own device, which must be current
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) throw Error(std::string("cudaGetDevice failed: ") + cudaGetErrorString(ce));
    if (dev != e->device)
      throw Error("the current CUDA device (" + std::to_string(dev) + ") is not the matrix's device (" +
                  std::to_string(e->device) + ")");
    if (dev < 0 || dev >= kMaxDevices) throw Error("device index out of range");
    void* scratch = scratch_address(dev);
    e->gemv_device_with_scratch(trans, alpha, x_dev, beta, y_dev, nrhs, (cudaStream_t)stream, scratch,
                                kNoAllocScratchBytes);
  } catch (const std::exception& ex) {
    return report_failure("hmat_b200_gemv_device_noalloc", ex.what());
  }
  return 0;
}
