// B200 engine: device residency and phase orchestration (see engine.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <tuple>
#include <type_traits>

#include "engine.h"
#include "gemv_plan.h"
#include "kernels.h"

#define HB_CUDA(x)                                                                                          \
  do {                                                                                                      \
    cudaError_t e_ = (x);                                                                                   \
    if (e_ != cudaSuccess) throw Error(std::string("CUDA error: ") + cudaGetErrorString(e_) + " in " #x); \
  } while (0)

namespace hmatb200 {
namespace {

template <typename X>
struct DevArray {
  X* p = nullptr;
  size_t n = 0;
  DevArray() = default;
  DevArray(const DevArray&) = delete;
  DevArray& operator=(const DevArray&) = delete;
  DevArray(DevArray&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  ~DevArray() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    release();
    if (count) HB_CUDA(cudaMalloc(&p, count * sizeof(X)));
    n = count;
  }
  void ensure(size_t count) {
    if (count > n) alloc(count);
  }
  void upload(const std::vector<X>& v, cudaStream_t s) {
    alloc(v.size());
    if (n) HB_CUDA(cudaMemcpyAsync(p, v.data(), n * sizeof(X), cudaMemcpyHostToDevice, s));
  }
  void swap(DevArray& o) {
    std::swap(p, o.p);
    std::swap(n, o.n);
  }
};

inline long long pad32(long long x) { return (x + 31) & ~31LL; }

// Workspace budget of the ACA phase (bytes); batches of admissible leaves are sized to it.
size_t workspace_budget() {
  const char* s = getenv("HMAT_B200_WORKSPACE_MB");
  long long mb = s ? atoll(s) : 8192;
  if (mb < 64) mb = 64;
  return (size_t)mb << 20;
}
// The tensor-memory y-phase kernel (map 4) is opt-in: HMAT_B200_TC_Y=1.  With 16
// right-hand sides each M=128, N=16, K=8 tf32 MMA costs about 90 cycles (measured), so the
// three-term split caps it below the warp-level tensor-core kernel's rate.
bool tc_y_enabled() {
  const char* s = getenv("HMAT_B200_TC_Y");
  return s && s[0] == '1';
}

// ACA autotuner.  Leaf-size buckets: leaves the warp-per-leaf kernel takes (m, n <= 64), then
// m + n below kAcaBigRows, below 4 kAcaBigRows, and above.  Shapes: warp per leaf, CTAs of 64,
// 128, 256 and 512 threads; each bucket has two candidates and a default (the measured best on
// the cylinder benchmark).  Every shape builds the same factors, so the choice only moves time.
enum AcaShape { kShapeWarp = 0, kShape64 = 1, kShape128 = 2, kShape256 = 3, kShape512 = 4 };
constexpr int kAcaBuckets = 4;
constexpr int kAcaShapes = 5;
constexpr int kShapeThreads[kAcaShapes] = {0, 64, 128, 256, 512};
constexpr int kAcaCand[kAcaBuckets][2] = {
    {kShapeWarp, kShape64}, {kShape128, kShape256}, {kShape128, kShape256}, {kShape256, kShape512}};
constexpr int kAcaDefault[kAcaBuckets] = {kShapeWarp, kShape128, kShape256, kShape256};
constexpr size_t kTuneRuns = 2 * kAcaBuckets;

int aca_bucket(int m, int n) {
  if (aca_warp_eligible(m, n)) return 0;
  const int len = m + n;
  return len < kAcaBigRows ? 1 : (len < 4 * kAcaBigRows ? 2 : 3);
}
// HMAT_B200_ACA_SHAPE=warp|64|128|256|512 forces one shape wherever it applies (the warp kernel
// only takes bucket 0); -1 when unset.
int forced_aca_shape() {
  const char* s = getenv("HMAT_B200_ACA_SHAPE");
  if (!s || !*s) return -1;
  if (!strcmp(s, "warp")) return kShapeWarp;
  const int t = atoi(s);
  return t == 64 ? kShape64 : t == 128 ? kShape128 : t == 256 ? kShape256 : t == 512 ? kShape512 : -1;
}
// HMAT_B200_ACA_TUNE=0 keeps the defaults; =2 samples every bucket of two leaves or more,
// however small, and neither reads nor writes the process's choices (a test mode).
int aca_tuning_mode() {
  const char* s = getenv("HMAT_B200_ACA_TUNE");
  if (!s || !*s) return 1;
  return s[0] == '0' ? 0 : (s[0] == '2' ? 2 : 1);
}
// Choices measured so far in this process, by (scalar type, kernel kind, epsilon decade,
// bucket).
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tune_cache;
// Gemv tuner choices of the process: (z chunk units, half-width y units) by (scalar type,
// height class of the output blocks).
std::map<std::tuple<int, int, int, int>, std::pair<int, bool>> g_gemv_tune_cache;

// HMAT_B200_GEMV_HALF_WARP_MAP=1 keeps the half-warp lane map (two column slices, 4 rows a lane)
// for the FP64 and complex output blocks of 33 to 64 rows, in place of lanes over rows.
bool gemv_half_warp_map() {
  const char* s = getenv("HMAT_B200_GEMV_HALF_WARP_MAP");
  return s && s[0] == '1';
}

// Bound of each gemv kernel's wait for a bulk copy (polls of the stage barrier).
// HMAT_B200_GEMV_WAIT_LIMIT changes it for the matrices created while it is set; a negative
// value makes every wait give up at once (a test hook: the kernels flag the product, let
// their copies land and stop, so that the status path is checked without a fault).
long long gemv_wait_limit() {
  const char* s = getenv("HMAT_B200_GEMV_WAIT_LIMIT");
  const long long v = (s && *s) ? atoll(s) : kGemvWaitLimit;
  return v < 0 ? -1 : (v < 1 ? 1 : v);
}

// Cap on the Jacobi sweeps of the truncation's core SVDs.  HMAT_B200_JACOBI_SWEEPS lowers it
// (a test hook: with one sweep most cores do not converge and the assembly reports it).
int jacobi_sweeps() {
  const char* s = getenv("HMAT_B200_JACOBI_SWEEPS");
  const int v = (s && *s) ? atoi(s) : kJacobiDefaultSweeps;
  return v < 1 ? 1 : v;
}

// Initial ACA rank capacity per leaf; leaves that reach it are rerun with twice as much.
int initial_kcap() {
  const char* s = getenv("HMAT_B200_ACA_KCAP");
  int k = s ? atoi(s) : 48;
  return k < 4 ? 4 : k;
}

// Output blocks of a cluster tree: its leaves in cluster order, cut into near-equal pieces
// of at most 128 rows (the row capacity of a gemv task).
struct Block {
  int off, len;
};
std::vector<Block> output_blocks(const ClusterTree& t) {
  std::vector<Block> b;
  for (int nd : t.leaf_nodes) {
    const int off = t.nodes[nd].offset, size = t.nodes[nd].size;
    if (size == 0) continue;
    const int nb = (size + 127) / 128, base = size / nb, rem = size % nb;
    int o = off;
    for (int i = 0; i < nb; ++i) {
      const int len = base + (i < rem ? 1 : 0);
      b.push_back(Block{o, len});
      o += len;
    }
  }
  return b;
}
// Blocks covering [off, off + len) (a union of blocks, since cluster ranges are).
std::pair<int, int> block_range(const std::vector<Block>& b, const std::vector<int>& starts, int off, int len) {
  int first = (int)(std::upper_bound(starts.begin(), starts.end(), off) - starts.begin()) - 1;
  int last = first;
  while (last < (int)b.size() && b[last].off < off + len) ++last;
  return {first, last};
}

template <typename T>
class Engine : public EngineBase {
  struct Piece;

 public:
  static constexpr int kPad = 16 / (int)sizeof(T) > 0 ? 16 / (int)sizeof(T) : 1;  // 16-byte alignment (elements)
  static long long padded(long long e) { return (e + kPad - 1) / kPad * kPad; }

  Engine(const ClusterTree* rows, const ClusterTree* cols, const BlockTree* bt) : R_(rows), C_(cols), bt_(bt) {
    HB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    HB_CUDA(cudaStreamCreateWithFlags(&stream2_, cudaStreamNonBlocking));
    HB_CUDA(cudaStreamCreateWithFlags(&stream3_, cudaStreamNonBlocking));
    HB_CUDA(cudaStreamCreateWithFlags(&stream4_, cudaStreamNonBlocking));
    HB_CUDA(cudaStreamCreateWithFlags(&stream5_, cudaStreamNonBlocking));
    for (auto& e : ev_) HB_CUDA(cudaEventCreate(&e));
    for (auto& e : tune_ev_) HB_CUDA(cudaEventCreate(&e));
    for (auto& e : fork_) HB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ranks.assign(bt_->leaves.size(), -1);
    for (size_t i = 0; i < bt_->leaves.size(); ++i)
      if (bt_->leaves[i].type == 1) ranks[i] = 0;
    rblocks_ = output_blocks(*R_);
    cblocks_ = output_blocks(*C_);
    for (auto& b : rblocks_) rstarts_.push_back(b.off);
    for (auto& b : cblocks_) cstarts_.push_back(b.off);
    HB_CUDA(cudaGetDevice(&device));
    err_.alloc(1);
    HB_CUDA(cudaMallocHost(&h_err_, sizeof(GemvStatus)));
    h_err_->failed = 0;
    h_err_->pad = 0;
    h_err_->wait_limit = gemv_wait_limit();
    HB_CUDA(cudaMemcpy(err_.p, h_err_, sizeof(GemvStatus), cudaMemcpyHostToDevice));
    preload_full_kernels<T>();
    preload_aca_kernels<T>();
    preload_truncate_kernels<T>();
    HB_CUDA(cudaGetLastError());
  }
  ~Engine() override {
    if (gexec_) cudaGraphExecDestroy(gexec_);
    for (auto& e : ev_) cudaEventDestroy(e);
    for (auto& e : fork_) cudaEventDestroy(e);
    for (auto& e : tune_ev_) cudaEventDestroy(e);
    if (h_err_) cudaFreeHost(h_err_);
    cudaStreamDestroy(stream2_);
    cudaStreamDestroy(stream3_);
    cudaStreamDestroy(stream4_);
    cudaStreamDestroy(stream5_);
    cudaStreamDestroy(stream_);
  }

  // ------------------------------------------------------------------------------
  void assemble(const AssemblyDesc& a, int method, double eps_aca, double eps_trunc, int svd_below) override {
    const int nr = R_->n, nc = C_->n;
    if ((long long)a.pts.size() != 3LL * nr || nr != nc)
      throw Error("assembly points must match the cluster trees (square matrix, same point count)");
    if (Traits<T>::is_complex != (a.kp.kind == kHelmholtzReg))
      throw Error("the Helmholtz kernel requires a complex value type and the real kernels a real one");
    if (method != 0 && method != 1) throw Error("only ACA+ and partial ACA compression run on the device");
    assembled = false;
    if (gexec_) {
      cudaGraphExecDestroy(gexec_);
      gexec_ = nullptr;
    }
    kp_ = a.kp;
    // a multi-strata kernel: a_0 .. a_{S-1}, w_0 .. w_{S-1}
    if (a.strata.size() % 2 || a.strata.size() > 2 * (size_t)kMaxStrata)
      throw Error("multi-strata kernel: 1 to " + std::to_string(kMaxStrata) + " strata");
    if (!a.strata.empty() && !a.param.empty())
      throw Error("a multi-strata kernel cannot take per-point parameters");
    strata_ = a.strata;
    const int nstrata = (int)strata_.size() / 2;
    kp_.nstrata = nstrata;
    kp_.strata = nullptr;
    if (nstrata) {
      d_strata_.upload(strata_, stream_);
      kp_.strata = d_strata_.p;
    }
    svd_below_ = svd_below;
    upload_points(a);
    const auto& L = bt_->leaves;
    const int nleaves = (int)L.size();
    piece_loff_.assign(nleaves, -1);
    times_ms[0] = times_ms[1] = times_ms[2] = 0;

    // ---- admissible leaves: ACA / SVD, truncation, compaction into pieces (stratum 0 of a
    // multi-strata kernel) ----
    assemble_rk(method, eps_aca, eps_trunc, svd_below, nstrata ? 0 : -1);

    // ---- final arena (the ranks fix the layout): full leaves evaluated in place, the Rk
    // factors moved from their pieces ----
    compute_layout();
    std::vector<FullLeafDesc> fd;
    std::vector<PanelDesc> fpanels;
    full_descs(fd, fpanels, nullptr);
    arena_.alloc((size_t)(layout_.total + 256));
    HB_CUDA(cudaMemsetAsync(arena_.p, 0, (size_t)layout_.total * sizeof(T), stream_));  // padding columns
    DevArray<FullLeafDesc> d_fd;
    DevArray<PanelDesc> d_fp;
    d_fd.upload(fd, stream_);
    d_fp.upload(fpanels, stream_);
    HB_CUDA(cudaEventRecord(ev_[0], stream_));
    launch_assemble_full<T>(d_fd.p, (int)fd.size(), d_fp.p, kp_, pts_, arena_.p, stream_);
    HB_CUDA(cudaGetLastError());
    HB_CUDA(cudaEventRecord(ev_[1], stream_));
    HB_CUDA(cudaStreamSynchronize(stream_));
    float ms = 0;
    HB_CUDA(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
    scatter_pieces(arena_.p, &ms);  // the compressed leaves placed in the arena, timed with them
    times_ms[0] = ms;
    pieces_.clear();
    // ---- the further strata, each joined to the factors the leaves hold ----
    for (int st = 1; st < nstrata; ++st) add_stratum(st, eps_aca, eps_trunc);
    build_plan();
    tune_gemv_plan();
    HB_CUDA(cudaStreamSynchronize(stream_));
    assembled = true;
  }

  // ------------------------------------------------------------------------------
  void gemv_device(char trans, const void* alpha, const void* x, const void* beta, void* y, int nrhs,
                   cudaStream_t user_stream) override {
    check_gemv_args(trans, nrhs);
    if (nrhs == 0) return;
    const T a = *(const T*)alpha, b = *(const T*)beta;
    xz_.ensure(xz_elems());
    GraphKey key(trans, nrhs, x, y);
    memcpy(key.ab, &a, sizeof(T));
    memcpy(key.ab + sizeof(T), &b, sizeof(T));
    if (!gexec_ || memcmp(&key, &gkey_, sizeof(GraphKey)) != 0) {
      if (gexec_) {
        cudaGraphExecDestroy(gexec_);
        gexec_ = nullptr;
      }
      cudaGraph_t g;
      HB_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      launch_gemv<T>(plan_, trans, nrhs, a, b, (const T*)x, (T*)y, xz_.p, err_.p, stream_);
      cudaError_t launch_err = cudaGetLastError();
      HB_CUDA(cudaStreamEndCapture(stream_, &g));
      HB_CUDA(launch_err);
      cudaError_t ie = cudaGraphInstantiate(&gexec_, g, 0);
      cudaGraphDestroy(g);
      HB_CUDA(ie);
      gkey_ = key;
    }
    cudaStream_t s = user_stream ? user_stream : stream_;
    HB_CUDA(cudaEventRecord(ev_[6], s));
    HB_CUDA(cudaGraphLaunch(gexec_, s));
    HB_CUDA(cudaEventRecord(ev_[7], s));
  }

  void gemv_host(char trans, const void* alpha, const void* x, const void* beta, void* y, int nrhs) override {
    check_gemv_args(trans, nrhs);
    if (nrhs == 0) return;
    const size_t n_in = trans == 'N' ? C_->n : R_->n, n_out = trans == 'N' ? R_->n : C_->n;
    stage_x_.ensure(n_in * nrhs);
    stage_y_.ensure(n_out * nrhs);
    HB_CUDA(cudaMemcpyAsync(stage_x_.p, x, n_in * nrhs * sizeof(T), cudaMemcpyHostToDevice, stream_));
    const T b = *(const T*)beta;
    if (!is_zero_val(b))
      HB_CUDA(cudaMemcpyAsync(stage_y_.p, y, n_out * nrhs * sizeof(T), cudaMemcpyHostToDevice, stream_));
    gemv_device(trans, alpha, stage_x_.p, beta, stage_y_.p, nrhs, stream_);
    HB_CUDA(cudaMemcpyAsync(y, stage_y_.p, n_out * nrhs * sizeof(T), cudaMemcpyDeviceToHost, stream_));
    // the status flag comes back with y (one synchronisation per call)
    HB_CUDA(cudaMemcpyAsync(&h_err_->failed, &err_.p->failed, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    HB_CUDA(cudaStreamSynchronize(stream_));
    HB_CUDA(cudaGetLastError());
    if (h_err_->failed) {
      clear_status(stream_);
      throw Error(kWaitGaveUp);
    }
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ev_[6], ev_[7]) == cudaSuccess) times_ms[3] = ms;
  }

  // ------------------------------------------------------------------------------
  long long leaf_payload(int leaf, void* out) override {
    if (!assembled || leaf < 0 || leaf >= (int)bt_->leaves.size()) return -1;
    const LeafInfo& L = bt_->leaves[leaf];
    if (layout_.first[leaf] < 0) return 0;
    const int k = ranks[leaf];
    const int w = L.type == 0 ? L.n : k;  // columns of a row panel
    auto br = block_range(rblocks_, rstarts_, L.row_off, L.m);
    T* o = (T*)out;
    std::vector<T> h;
    for (int b = br.first; b < br.second; ++b) {  // row panels -> column-major m x w
      const int rs = rblocks_[b].off - L.row_off, len = rblocks_[b].len;
      h.resize((size_t)len * w);
      HB_CUDA(cudaMemcpy(h.data(), arena_.p + layout_.panel[layout_.first[leaf] + (b - br.first)],
                         h.size() * sizeof(T), cudaMemcpyDeviceToHost));
      for (int j = 0; j < w; ++j)
        for (int i = 0; i < len; ++i) o[(size_t)rs + i + (size_t)j * L.m] = h[i + (size_t)j * len];
    }
    if (L.type == 0) return (long long)L.m * L.n;
    h.resize((size_t)k * L.n);
    HB_CUDA(cudaMemcpy2D(h.data(), (size_t)k * sizeof(T), arena_.p + layout_.bt[leaf],
                         (size_t)layout_.bt_ld[leaf] * sizeof(T), (size_t)k * sizeof(T), L.n, cudaMemcpyDeviceToHost));
    T* Bo = o + (size_t)L.m * k;  // B^T (k x n) -> B (n x k)
    for (int j = 0; j < L.n; ++j)
      for (int l = 0; l < k; ++l) Bo[j + (size_t)l * L.n] = h[l + (size_t)j * k];
    return (long long)k * (L.m + L.n);
  }

  void payload_layout(long long* offsets, long long* total) override {
    long long acc = 0;
    const auto& L = bt_->leaves;
    for (size_t i = 0; i < L.size(); ++i) {
      if (offsets) offsets[i] = acc;
      if (L[i].type == 0) acc += (long long)L[i].m * L[i].n;
      else if (ranks[i] > 0) acc += (long long)ranks[i] * (L[i].m + L[i].n);
    }
    if (total) *total = acc;
  }

  void leaf_gradients(const void* x, const void* r, int nrhs, void* grad, bool accumulate,
                      cudaStream_t user_stream) override {
    if (!assembled) throw Error("matrix is not assembled");
    if (Traits<T>::is_complex) throw Error("leaf gradients are implemented for real value types");
    if (nrhs < 1 || nrhs > 16) throw Error("leaf gradients take 1 to 16 right-hand sides");
    check_device();
    xz_.ensure(xz_elems());
    rz_.ensure(xz_elems());
    cudaStream_t s = user_stream ? user_stream : stream_;
    launch_leaf_gradients<T>(plan_, nrhs, (const T*)x, (const T*)r, xz_.p, rz_.p, (T*)grad, (T*)grad, accumulate,
                             err_.p, s);
    HB_CUDA(cudaGetLastError());
  }

  void gemv_adjoint(const void* x, const void* r, int nrhs, void* dx, void* grad, bool accumulate,
                    cudaStream_t user_stream) override {
    if (!assembled) throw Error("matrix is not assembled");
    if (Traits<T>::is_complex) throw Error("the adjoint is implemented for real value types");
    if (nrhs < 1 || nrhs > 16) throw Error("the adjoint takes 1 to 16 right-hand sides");
    check_device();
    xz_.ensure(xz_elems());
    rz_.ensure(xz_elems());
    cudaStream_t s = user_stream ? user_stream : stream_;
    launch_gemv_adjoint<T>(plan_, nrhs, (const T*)x, (const T*)r, (T*)dx, xz_.p, rz_.p, (T*)grad, (T*)grad, accumulate,
                           err_.p, s);
    HB_CUDA(cudaGetLastError());
  }

  void load_leaves(const int* rk_in, const void* canonical) override {
    const auto& L = bt_->leaves;
    const int nleaves = (int)L.size();
    for (int i = 0; i < nleaves; ++i) {
      if (L[i].type == 0 && rk_in[i] != -1) throw Error("stored data: rank given for a full leaf");
      if (L[i].type == 1 && (rk_in[i] < 0 || rk_in[i] > std::min(L[i].m, L[i].n)))
        throw Error("stored data: rank out of range");
    }
    assembled = false;
    if (gexec_) {
      cudaGraphExecDestroy(gexec_);
      gexec_ = nullptr;
    }
    ranks.assign(rk_in, rk_in + nleaves);
    // the permutations the gemv gathers and scatters with (assemble uploads them with the
    // points; a loaded matrix has no points)
    d_perm_rows_.upload(R_->perm, stream_);
    d_perm_cols_.upload(C_->perm, stream_);
    std::vector<long long> goff(nleaves);
    long long total = 0;
    payload_layout(goff.data(), &total);
    compute_layout();
    // full leaves: canonical m x n into their row panels
    std::vector<FullLeafDesc> fd;
    std::vector<long long> fgoff;
    std::vector<PanelDesc> fpanels;
    full_descs(fd, fpanels, &fgoff, &goff);
    // Rk leaves: canonical A (m x k) and B (n x k) into the A panels and B^T
    std::vector<RkLeafDesc> rd;
    std::vector<int> rk;
    std::vector<RkStoreDesc> store;
    std::vector<PanelDesc> panels;
    for (int i = 0; i < nleaves; ++i) {
      const int k = ranks[i];
      if (L[i].type != 1 || k <= 0) continue;
      RkLeafDesc d;
      d.row_off = L[i].row_off;
      d.m = L[i].m;
      d.col_off = L[i].col_off;
      d.n = L[i].n;
      d.ws_off = goff[i];
      d.fl_off = 0;
      d.kcap = k;
      d.pad = 0;
      rd.push_back(d);
      rk.push_back(k);
      store.push_back(rk_store(i, panels));
    }
    arena_.alloc((size_t)(layout_.total + 256));
    HB_CUDA(cudaMemsetAsync(arena_.p, 0, (size_t)layout_.total * sizeof(T), stream_));
    DevArray<T> src;
    src.alloc((size_t)std::max(total, 1LL));
    if (total) HB_CUDA(cudaMemcpyAsync(src.p, canonical, total * sizeof(T), cudaMemcpyHostToDevice, stream_));
    DevArray<FullLeafDesc> d_fd;
    DevArray<long long> d_fgoff;
    DevArray<PanelDesc> d_fp, d_panels;
    DevArray<RkLeafDesc> d_rd;
    DevArray<int> d_rk;
    DevArray<RkStoreDesc> d_store;
    d_fd.upload(fd, stream_);
    d_fgoff.upload(fgoff, stream_);
    d_fp.upload(fpanels, stream_);
    d_rd.upload(rd, stream_);
    d_rk.upload(rk, stream_);
    d_store.upload(store, stream_);
    d_panels.upload(panels, stream_);
    launch_full_from_canonical<T>(d_fd.p, d_fgoff.p, (int)fd.size(), d_fp.p, src.p, arena_.p, stream_);
    HB_CUDA(cudaGetLastError());
    launch_compact<T>(d_rd.p, (int)rd.size(), src.p, d_rk.p, d_store.p, d_panels.p, arena_.p, stream_);
    HB_CUDA(cudaGetLastError());
    HB_CUDA(cudaStreamSynchronize(stream_));
    build_plan();
    tune_gemv_plan();
    HB_CUDA(cudaStreamSynchronize(stream_));
    for (int i = 0; i < 4; ++i) times_ms[i] = 0;
    assembled = true;
  }

  // HMatrix::truncate (h_matrix.cpp:2107-2123): every Rk leaf re-truncated at eps with the
  // assembly's truncation kernels, then the arena and the gemv schedule rebuilt.
  void retruncate(double eps) override {
    if (!assembled) throw Error("matrix not assembled");
    check_device();
    HB_CUDA(set_jacobi_max_sweeps(jacobi_sweeps()));
    const auto& L = bt_->leaves;
    const int nleaves = (int)L.size();
    double saved[4];
    for (int i = 0; i < 4; ++i) saved[i] = times_ms[i];
    std::vector<RkJob> queue;
    for (int i = 0; i < nleaves; ++i)
      if (L[i].type == 1 && ranks[i] > 0) {
        RkJob j;
        j.leaf = i;
        j.kcap = ranks[i];
        j.svd = false;
        queue.push_back(j);
      }
    piece_of_.assign(nleaves, -1);
    piece_loff_.assign(nleaves, -1);
    pieces_.clear();
    const size_t budget = workspace_budget();
    size_t pos = 0;
    while (pos < queue.size()) {
      std::vector<RkJob> batch, retry;
      size_t bytes = 0;
      while (pos < queue.size()) {
        const LeafInfo& l = L[queue[pos].leaf];
        size_t b = (size_t)pad32(rk_slot_elems(l.m, l.n, queue[pos].kcap)) * sizeof(T) + l.m + l.n;
        if (!batch.empty() && bytes + b > budget) break;
        bytes += b;
        batch.push_back(queue[pos++]);
      }
      run_batch(batch, eps, eps, retry, arena_.p);  // unpacks with the current layout
      if (!retry.empty()) throw Error("re-truncation: unexpected capacity retry");
    }
    rebuild_arena();
    if (gexec_) {
      cudaGraphExecDestroy(gexec_);
      gexec_ = nullptr;
    }
    build_plan();
    tune_gemv_plan();
    HB_CUDA(cudaStreamSynchronize(stream_));
    for (int i = 0; i < 4; ++i) times_ms[i] = saved[i];
  }

  void profile_gemv(char trans, const void* x, void* y, int nrhs, double* ms3, double* bytes3) override {
    check_gemv_args(trans, nrhs);
    if (nrhs < 1 || nrhs > 16) throw Error("profile_gemv takes 1 to 16 right-hand sides");
    xz_.ensure(xz_elems());
    GemvTiming tm;
    for (int i = 0; i < 4; ++i) HB_CUDA(cudaEventCreate(&tm.ev[i]));
    launch_gemv<T>(plan_, trans, nrhs, one<T>(), zero<T>(), (const T*)x, (T*)y, xz_.p, err_.p, stream_, &tm);
    cudaError_t le = cudaGetLastError();
    cudaError_t se = cudaStreamSynchronize(stream_);
    float a = 0, b = 0, c = 0;
    if (le == cudaSuccess && se == cudaSuccess) {
      cudaEventElapsedTime(&a, tm.ev[0], tm.ev[1]);
      cudaEventElapsedTime(&b, tm.ev[1], tm.ev[2]);
      cudaEventElapsedTime(&c, tm.ev[2], tm.ev[3]);
    }
    for (int i = 0; i < 4; ++i) cudaEventDestroy(tm.ev[i]);
    HB_CUDA(le);
    HB_CUDA(se);
    check_err_flag();
    ms3[0] = a;
    ms3[1] = b;
    ms3[2] = c;
    const double s = sizeof(T);
    const auto& L = bt_->leaves;
    double full = 0, fa = 0, fb = 0;
    for (size_t i = 0; i < L.size(); ++i) {
      if (L[i].type == 0 && layout_.first[i] >= 0) full += (double)L[i].m * L[i].n;
      if (L[i].type == 1 && ranks[i] > 0) {
        fa += (double)L[i].m * ranks[i];
        fb += (double)L[i].n * ranks[i];
      }
    }
    const double n_in = trans == 'N' ? C_->n : R_->n, n_out = trans == 'N' ? R_->n : C_->n;
    bytes3[0] = 2.0 * n_in * nrhs * s;
    bytes3[1] = (trans == 'N' ? fb : fa) * s;
    bytes3[2] = (full + (trans == 'N' ? fa : fb)) * s + n_out * nrhs * s;
  }

  size_t gemv_scratch_bytes() const override { return xz_elems() * sizeof(T); }
  int gemv_launches(char trans, int nrhs) const override {
    if (!assembled) throw Error("matrix not assembled");
    return gemv_launch_count(plan_, trans, nrhs, (int)sizeof(T));
  }

  void gemv_device_with_scratch(char trans, const void* alpha, const void* x, const void* beta, void* y, int nrhs,
                                cudaStream_t stream, void* scratch, size_t scratch_bytes) override {
    check_gemv_args(trans, nrhs);
    if (nrhs == 0) return;
    if (gemv_scratch_bytes() > scratch_bytes) throw Error("scratch buffer too small for this matrix");
    cudaStream_t s = stream ? stream : stream_;
    // the status flag is the matrix's own (allocated with the engine), read by gemv_status
    launch_gemv<T>(plan_, trans, nrhs, *(const T*)alpha, *(const T*)beta, (const T*)x, (T*)y, (T*)scratch, err_.p,
                   s);
    HB_CUDA(cudaGetLastError());
  }

  int gemv_status(cudaStream_t user_stream) override {
    check_device();
    cudaStream_t s = user_stream ? user_stream : stream_;
    HB_CUDA(cudaMemcpyAsync(&h_err_->failed, &err_.p->failed, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    const int failed = h_err_->failed;
    if (failed == 2)  // a unit that failed its copy checks (index in the second word)
      fprintf(stderr, "gemv: unit %d of the schedule failed its copy checks and was skipped\n", h_err_->pad);
    if (failed) clear_status(s);
    return failed;
  }

 private:
  struct GraphKey {
    char trans;
    int nrhs;
    const void* x;
    void* y;
    unsigned char ab[2 * sizeof(cdouble)];
    GraphKey() { memset(this, 0, sizeof(*this)); }
    GraphKey(char t, int n, const void* xx, void* yy) {
      memset(this, 0, sizeof(*this));
      trans = t;
      nrhs = n;
      x = xx;
      y = yy;
    }
  };

  size_t xz_elems() const {
    return (size_t)std::max(plan_.xz_rows, 1LL) * gemv_rhs_stride((int)sizeof(T), 16);
  }

  static constexpr const char* kWaitGaveUp =
      "gemv: a kernel's wait for a bulk copy gave up, in this product or an earlier device product of this matrix "
      "(its result is not valid)";

  // The engine's streams, arena and status block live on the device that was current when
  // the matrix was created; products must be issued with that device current.
  void check_device() const {
    int d = -1;
    HB_CUDA(cudaGetDevice(&d));
    if (d != device)
      throw Error("the current CUDA device (" + std::to_string(d) + ") is not the matrix's device (" +
                  std::to_string(device) + ")");
  }

  void clear_status(cudaStream_t s) {
    h_err_->failed = 0;
    h_err_->pad = 0;
    HB_CUDA(cudaMemsetAsync(&err_.p->failed, 0, 2 * sizeof(int), s));
    HB_CUDA(cudaStreamSynchronize(s));
  }

  void check_gemv_args(char trans, int nrhs) {
    if (!assembled) throw Error("matrix is not assembled");
    check_device();
    if (trans != 'N' && trans != 'T' && trans != 'C') throw Error("gemv: trans must be 'N', 'T' or 'C'");
    if (nrhs < 0) throw Error("gemv: negative number of right-hand sides");
  }

  void check_err_flag() {
    int e = 0;
    HB_CUDA(cudaMemcpy(&e, &err_.p->failed, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
      clear_status(stream_);
      throw Error(kWaitGaveUp);
    }
  }

  void upload_points(const AssemblyDesc& a) {
    const int nr = R_->n, nc = C_->n;
    std::vector<double> h(3 * (size_t)nr + 3 * (size_t)nc);
    for (int i = 0; i < nr; ++i)
      for (int d = 0; d < 3; ++d) h[(size_t)d * nr + i] = a.pts[3 * (size_t)R_->perm[i] + d];
    double* hc = h.data() + 3 * (size_t)nr;
    for (int i = 0; i < nc; ++i)
      for (int d = 0; d < 3; ++d) hc[(size_t)d * nc + i] = a.pts[3 * (size_t)C_->perm[i] + d];
    d_pts_.upload(h, stream_);
    d_perm_rows_.upload(R_->perm, stream_);
    d_perm_cols_.upload(C_->perm, stream_);
    pts_.rx = d_pts_.p;
    pts_.ry = d_pts_.p + nr;
    pts_.rz = d_pts_.p + 2 * (size_t)nr;
    pts_.cx = d_pts_.p + 3 * (size_t)nr;
    pts_.cy = pts_.cx + nc;
    pts_.cz = pts_.cx + 2 * (size_t)nc;
    pts_.rid = d_perm_rows_.p;
    pts_.cid = d_perm_cols_.p;
    pts_.rprm = nullptr;
    if (!a.param.empty()) {
      // per-point kernel parameter, taken from the row point (cluster order)
      if ((long long)a.param.size() != nr) throw Error("one kernel parameter per point is needed");
      std::vector<double> hp(nr);
      for (int i = 0; i < nr; ++i) hp[i] = a.param[R_->perm[i]];
      d_prm_.upload(hp, stream_);
      pts_.rprm = d_prm_.p;
    }
  }

  struct RkJob {
    int leaf;
    int kcap;
    bool svd;
    bool cta = false;   // ACA on the CTA-per-leaf kernel (a retry after a capacity overflow)
    int kcur = 0;       // a further stratum: the rank the leaf holds in the arena
    bool pass = false;  // a further stratum: no ACA, the held factors kept as they are
  };
  struct Piece {
    DevArray<T> arena;
    long long elems = 0;
  };

  // Runs ACA (or the dense-SVD fill) and the truncation on one batch of admissible
  // leaves; leaves that ran out of rank capacity are returned in `retry`, the others are
  // compacted (A as row panels, B transposed) into a new piece.
  // With `src` set, the leaves are already assembled: their factors are unpacked from the
  // arena `src` (rank = kcap) instead of being computed, then truncated at eps_trunc.
  // With a multi-strata kernel, `stratum` >= 0 is the stratum whose ACA runs (the plain kernel
  // with the stratum's parameter; A then scaled by its weight).  Stratum 0 is compressed as a
  // plain kernel; a further stratum (src = the arena) is joined to the factors the leaves hold
  // (kcur columns): concatenated and truncated, or, once the summed rank reaches min(m, n),
  // summed as a full block and compressed by SVD, then truncated (compression.cpp:745-773,
  // rk_matrix.cpp:846-1009).  The dense-SVD jobs compress the sum of the strata.
  void run_batch(const std::vector<RkJob>& jobs_in, double eps_aca, double eps_trunc, std::vector<RkJob>& retry,
                 const T* src = nullptr, int stratum = -1) {
    const auto& L = bt_->leaves;
    std::vector<RkJob> jobs = jobs_in;  // a further stratum turns its dense sums into SVD jobs
    const bool add_stratum = stratum >= 1;
    if (add_stratum && !src) throw Error("stratum assembly without the arena");
    const KernelParams kp_aca = stratum >= 0 ? stratum_kp(stratum) : kp_;
    const int nb = (int)jobs.size();
    std::vector<RkLeafDesc> desc(nb);
    long long ws = 0, fl = 0;
    int max_m = 1, max_n = 1, max_cap = 1;
    for (int b = 0; b < nb; ++b) {
      const LeafInfo& l = L[jobs[b].leaf];
      RkLeafDesc& d = desc[b];
      d.row_off = l.row_off;
      d.m = l.m;
      d.col_off = l.col_off;
      d.n = l.n;
      d.kcap = jobs[b].kcap;
      d.ws_off = ws;
      d.fl_off = fl;
      d.pad = 0;
      ws += pad32(rk_slot_elems(l.m, l.n, d.kcap));
      fl += l.m + l.n;
      max_m = std::max(max_m, l.m);
      max_n = std::max(max_n, l.n);
      max_cap = std::max(max_cap, d.kcap);
    }
    // ACA shape of each leaf: the autotuner's choice for its size bucket; capacity retries run
    // on CTAs (512 threads from m + n >= kAcaBigRows, where the retried ranks are high).
    std::vector<int> svd_order, bucket_list[kAcaBuckets], shape_order[kAcaShapes];
    auto cost = [&](int b) { return (double)(desc[b].m + desc[b].n) * std::min(desc[b].m, desc[b].n); };
    auto by_cost = [&](std::vector<int>& v) {
      std::stable_sort(v.begin(), v.end(), [&](int x, int y) { return cost(x) > cost(y); });
    };
    const int forced = forced_aca_shape();
    if (!src || add_stratum) {
      for (int b = 0; b < nb; ++b) {
        if (jobs[b].pass) continue;
        if (jobs[b].svd)
          svd_order.push_back(b);
        else if (jobs[b].cta)
          shape_order[forced > kShapeWarp ? forced
                                          : (desc[b].m + desc[b].n >= kAcaBigRows ? kShape512 : kShape128)]
              .push_back(b);
        else
          bucket_list[aca_bucket(desc[b].m, desc[b].n)].push_back(b);
      }
    }
    for (auto& v : bucket_list) by_cost(v);

    // Autotuner: a bucket without a choice yet (for this scalar type, kernel kind and epsilon
    // decade) runs one or two waves of each candidate shape on samples spread evenly over its
    // cost-sorted leaves and dealt alternately, so that both samples are alike, timed alone on
    // stream_; the shape with the most leaf cost per millisecond takes the rest of the bucket
    // and is kept for the process.  The sampled leaves are compressed for good.
    struct TuneRun {
      int bucket, shape;
      size_t begin, count;
      double cost;
    };
    std::vector<TuneRun> runs;
    std::vector<int> tune_order;
    int choice[kAcaBuckets];
    const int eps_dec = (int)std::floor(std::log10(std::max(eps_aca, 1e-300)) + 1e-9);
    auto tune_key = [&](int bk) {
      return std::make_tuple((int)sizeof(T) * 2 + (Traits<T>::is_complex ? 1 : 0), (int)kp_.kind, eps_dec, bk);
    };
    for (int bk = 0; bk < kAcaBuckets; ++bk) {
      choice[bk] = kAcaDefault[bk];
      const auto& lst = bucket_list[bk];
      if (lst.empty()) continue;
      aca_shape[bk] = kShapeThreads[choice[bk]];
      if (forced >= 0) {
        if (forced != kShapeWarp || bk == 0) choice[bk] = forced;
        continue;
      }
      const int mode = aca_tuning_mode();
      if (mode == 0) continue;
      if (mode == 1) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tune_cache.find(tune_key(bk));
        if (it != g_tune_cache.end()) {
          choice[bk] = it->second;
          if (aca_tuned[bk] != 1) aca_tuned[bk] = 2;  // an earlier batch of this assembly may have measured it
          continue;
        }
      }
      long long conc[2], wave = 0;
      for (int v = 0; v < 2; ++v) {
        conc[v] = aca_concurrency<T>(kShapeThreads[kAcaCand[bk][v]], max_cap);
        wave += conc[v];
      }
      const long long n = (long long)lst.size();
      // only where the samples are at most a thirty-second of the bucket: each serial run
      // lasts as long as its slowest leaf, about 0.5 ms for a bucket's largest leaves, which
      // only a bucket of many waves amortises
      const int waves = n >= 64 * wave ? 2 : (n >= 32 * wave ? 1 : 0);
      size_t ns = 0;
      if (waves)
        ns = (size_t)(waves * wave);
      else if (mode == 2 && n >= 2)
        ns = (size_t)(n / 2);
      else
        continue;
      // the samples are spread evenly over the cost-sorted bucket (the largest leaves alone
      // misjudge a bucket of mostly small ones); sample leaf i goes to the shape furthest below
      // its share (shares in proportion to the leaves each shape has in flight)
      std::vector<int> samp[2], rest_bk;
      std::vector<char> taken(lst.size(), 0);
      for (size_t i = 0; i < ns; ++i) taken[(size_t)((double)i * lst.size() / ns)] = 1;
      for (size_t i = 0; i < lst.size(); ++i) {
        if (!taken[i]) {
          rest_bk.push_back(lst[i]);
          continue;
        }
        const int v = (double)samp[0].size() * conc[1] <= (double)samp[1].size() * conc[0] ? 0 : 1;
        samp[v].push_back(lst[i]);
      }
      bucket_list[bk].swap(rest_bk);  // the rest, still in cost order
      for (int v = 0; v < 2; ++v) {
        double c = 0;
        for (int b : samp[v]) c += cost(b);
        runs.push_back(TuneRun{bk, kAcaCand[bk][v], tune_order.size(), samp[v].size(), c});
        tune_order.insert(tune_order.end(), samp[v].begin(), samp[v].end());
      }
    }
    if (runs.size() > kTuneRuns) throw Error("ACA autotuner: too many sample runs");

    DevArray<RkLeafDesc> d_desc;
    d_desc.upload(desc, stream_);
    DevArray<T> d_ws;
    d_ws.alloc((size_t)ws);
    DevArray<unsigned char> d_flags;
    d_flags.alloc((size_t)std::max(fl, 1LL));
    DevArray<int> d_ranks, d_status, d_counter, d_tune_order, d_svd_order, d_shape_order[kAcaShapes];
    d_ranks.alloc(nb);
    d_status.alloc(nb);
    d_counter.alloc(kAcaShapes + kTuneRuns);
    HB_CUDA(cudaMemsetAsync(d_ranks.p, 0, nb * sizeof(int), stream_));
    HB_CUDA(cudaMemsetAsync(d_status.p, 0, nb * sizeof(int), stream_));
    HB_CUDA(cudaMemsetAsync(d_counter.p, 0, (kAcaShapes + kTuneRuns) * sizeof(int), stream_));
    d_tune_order.upload(tune_order, stream_);
    d_svd_order.upload(svd_order, stream_);
    for (auto& d : d_shape_order) d.alloc((size_t)nb);
    // the rest of each bucket goes to its chosen shape; without sample runs the lists are
    // complete (and on the device) before the timed region
    auto finish_shapes = [&]() {
      for (int bk = 0; bk < kAcaBuckets; ++bk) {
        if (bucket_list[bk].empty()) continue;
        aca_shape[bk] = kShapeThreads[choice[bk]];
        shape_order[choice[bk]].insert(shape_order[choice[bk]].end(), bucket_list[bk].begin(),
                                       bucket_list[bk].end());
      }
      for (int sh = 0; sh < kAcaShapes; ++sh) {
        by_cost(shape_order[sh]);
        if (!shape_order[sh].empty())
          HB_CUDA(cudaMemcpyAsync(d_shape_order[sh].p, shape_order[sh].data(), shape_order[sh].size() * sizeof(int),
                                  cudaMemcpyHostToDevice, stream_));
      }
    };
    if (runs.empty()) finish_shapes();
    HB_CUDA(cudaStreamSynchronize(stream_));

    if (src && !add_stratum) {
      // rank = kcap: the stored factors, unpacked from their panels
      std::vector<int> k0(nb);
      std::vector<RkStoreDesc> ostore(nb);
      std::vector<PanelDesc> opanels;
      for (int b = 0; b < nb; ++b) {
        k0[b] = jobs[b].kcap;
        ostore[b] = rk_store(jobs[b].leaf, opanels);  // the stored leaf in the current layout
      }
      d_ranks.upload(k0, stream_);
      DevArray<RkStoreDesc> d_ostore;
      DevArray<PanelDesc> d_opanels;
      d_ostore.upload(ostore, stream_);
      d_opanels.upload(opanels, stream_);
      launch_unpack<T>(d_desc.p, nb, d_ranks.p, d_ostore.p, d_opanels.p, src, d_ws.p, stream_);
      HB_CUDA(cudaGetLastError());
      HB_CUDA(cudaStreamSynchronize(stream_));
    }
    auto launch_shape = [&](int shape, const int* order, int count, int* counter, cudaStream_t s) {
      if (count <= 0) return;
      if (shape == kShapeWarp)
        launch_aca_warp<T>(d_desc.p, order, count, kp_aca, pts_, eps_aca, d_ws.p, d_ranks.p, d_status.p, counter,
                           max_cap, s);
      else
        launch_aca<T>(d_desc.p, order, count, kp_aca, pts_, eps_aca, d_ws.p, d_flags.p, d_ranks.p, d_status.p,
                      counter, max_cap, aca_concurrency<T>(kShapeThreads[shape], max_cap), s, kShapeThreads[shape]);
      HB_CUDA(cudaGetLastError());
    };
    HB_CUDA(cudaEventRecord(ev_[2], stream_));
    if (!runs.empty()) {
      for (size_t r = 0; r < runs.size(); ++r) {
        HB_CUDA(cudaEventRecord(tune_ev_[2 * r], stream_));
        launch_shape(runs[r].shape, d_tune_order.p + runs[r].begin, (int)runs[r].count,
                     d_counter.p + kAcaShapes + r, stream_);
        HB_CUDA(cudaEventRecord(tune_ev_[2 * r + 1], stream_));
      }
      HB_CUDA(cudaStreamSynchronize(stream_));
      double best[kAcaBuckets] = {0, 0, 0, 0};
      for (size_t r = 0; r < runs.size(); ++r) {
        float ms = 0;
        HB_CUDA(cudaEventElapsedTime(&ms, tune_ev_[2 * r], tune_ev_[2 * r + 1]));
        const int bk = runs[r].bucket;
        const double rate = runs[r].cost / std::max((double)ms, 1e-6);
        aca_rate[bk][runs[r].shape] = rate;
        if (rate > best[bk]) {
          best[bk] = rate;
          choice[bk] = runs[r].shape;
        }
      }
      const bool keep = aca_tuning_mode() == 1;
      std::lock_guard<std::mutex> g(g_tune_mu);
      for (const auto& r : runs) {
        if (keep) g_tune_cache[tune_key(r.bucket)] = choice[r.bucket];
        aca_tuned[r.bucket] = 1;
      }
    }
    if (!runs.empty()) finish_shapes();
    // each shape on its own stream, beside the others: warp per leaf, 64, 256 and 512 on the
    // side streams, 128 and the dense-SVD fills on stream_
    const cudaStream_t side[kAcaShapes] = {stream2_, stream4_, stream_, stream5_, stream3_};
    for (int sh = 0; sh < kAcaShapes; ++sh) {
      if (shape_order[sh].empty() || side[sh] == stream_) continue;
      HB_CUDA(cudaEventRecord(fork_[2 * sh], stream_));
      HB_CUDA(cudaStreamWaitEvent(side[sh], fork_[2 * sh], 0));
      launch_shape(sh, d_shape_order[sh].p, (int)shape_order[sh].size(), d_counter.p + sh, side[sh]);
      HB_CUDA(cudaEventRecord(fork_[2 * sh + 1], side[sh]));
    }
    launch_shape(kShape128, d_shape_order[kShape128].p, (int)shape_order[kShape128].size(), d_counter.p + kShape128,
                 stream_);
    if (!svd_order.empty()) {
      launch_dense_to_rk<T>(d_desc.p, d_svd_order.p, (int)svd_order.size(), kp_, pts_, d_ws.p, d_ranks.p,
                            d_status.p, stream_);
      HB_CUDA(cudaGetLastError());
    }
    for (int sh = 0; sh < kAcaShapes; ++sh)
      if (!shape_order[sh].empty() && side[sh] != stream_) HB_CUDA(cudaStreamWaitEvent(stream_, fork_[2 * sh + 1], 0));
    HB_CUDA(cudaEventRecord(ev_[3], stream_));
    std::vector<int> h_status(nb), h_ranks(nb);
    HB_CUDA(cudaMemcpyAsync(h_status.data(), d_status.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    HB_CUDA(cudaMemcpyAsync(h_ranks.data(), d_ranks.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    HB_CUDA(cudaStreamSynchronize(stream_));
    float ms = 0;
    HB_CUDA(cudaEventElapsedTime(&ms, ev_[2], ev_[3]));
    times_ms[1] += ms;
    if (stratum >= 0) join_stratum(stratum, jobs, desc, d_desc, d_ws, d_ranks, h_status, h_ranks, src);

    std::vector<int> good;
    int max_k = 1;
    for (int b = 0; b < nb; ++b) {
      if (h_status[b] == kLeafAcaCapacity) {
        const LeafInfo& l = L[jobs[b].leaf];
        RkJob j = jobs[b];
        j.kcap = std::min(std::min(l.m, l.n), 2 * j.kcap);
        j.cta = true;
        retry.push_back(j);
        h_ranks[b] = 0;
        continue;
      }
      if (h_status[b] != kLeafOk)
        throw Error("device compression failed on a leaf (status " + std::to_string(h_status[b]) + ")");
      if (h_ranks[b] > 0 && !jobs[b].pass) good.push_back(b);
      max_k = std::max(max_k, h_ranks[b]);
    }
    auto tcost = [&](int b) { return (double)(desc[b].m + desc[b].n) * h_ranks[b] * h_ranks[b]; };
    std::stable_sort(good.begin(), good.end(), [&](int x, int y) { return tcost(x) > tcost(y); });

    typedef typename Traits<T>::wide W;
    DevArray<W> d_scratch, d_tri, d_maps;
    DevArray<int> d_good, d_svd_good;
    DevArray<TsItem> d_ts_seg[4], d_ts_stack[4];
    DevArray<TsCore> d_ts_core[4];
    long long slab = 0, grid = 0;
    std::vector<int> svd_good, large;
    std::vector<TsItem> ts_seg[4], ts_stack[4];
    std::vector<TsCore> ts_core[4];
    bool any_ts = false;
    // high-rank leaves: the same phases with a CTA per item
    std::vector<TsItem> tb_seg, tb_stack;
    std::vector<TsCore> tb_core;
    DevArray<TsItem> d_tb_seg, d_tb_stack;
    DevArray<TsCore> d_tb_core;
    DevArray<W> d_tb_tri, d_tb_maps, d_tb_scratch;
    long long tb_slab = 0;
    int tb_grid = 0;
    if (!good.empty()) {
      // Leaves up to rank ts_kmax go to the tall-skinny phases (row segments of A and B
      // reduced to triangles, stacks of triangles reduced again, core, apply), higher ranks
      // to the same phases with a CTA per item; the dense-SVD jobs, whose rank is only known
      // on the device, to the CTA-per-leaf kernel.
      int big_m = 1, big_n = 1, big_k = 1;
      long long tri_n = 0, map_n = 0, tb_tri = 0, tb_map = 0;
      int tb_rows = 1, tb_k = 1;
      const int kmax = ts_kmax<T>();
      for (int b : good) {
        if (jobs[b].svd) {
          large.push_back(b);
          big_m = std::max(big_m, desc[b].m);
          big_n = std::max(big_n, desc[b].n);
          big_k = std::max(big_k, h_ranks[b]);
          continue;
        }
        const int K = ts_bucket(h_ranks[b], kmax);
        if (!K) {
          // segments of at least k rows (the last one takes the remainder)
          const RkLeafDesc& d = desc[b];
          const int k = h_ranks[b];
          TsCore c{};
          c.leaf = b;
          c.k = k;
          for (int side = 0; side < 2; ++side) {
            const int len = side ? d.n : d.m;
            const long long base = d.ws_off + (side ? (long long)d.m * d.kcap : 0);
            const int S = std::max(kTsSegRows, k);
            const int p = std::max(1, len / S);
            const long long fin = tb_tri, mo = tb_map;
            tb_tri += (long long)k * k;
            tb_map += (long long)k * k;
            (side ? c.rb : c.ra) = fin;
            (side ? c.mb : c.ma) = mo;
            long long stk = 0;
            if (p > 1) {
              stk = tb_tri;
              tb_tri += (long long)p * k * k;
            }
            for (int sg = 0; sg < p; ++sg) {
              TsItem it{};
              it.src = base + (long long)sg * S;
              it.rows = sg == p - 1 ? len - sg * S : S;
              it.ld = len;
              it.r_out = p == 1 ? fin : stk + (long long)sg * k;
              it.ld_r = p == 1 ? k : p * k;
              it.map = mo;
              it.leaf = b;
              it.k = k;
              tb_rows = std::max(tb_rows, it.rows);
              tb_seg.push_back(it);
            }
            if (p > 1) {
              TsItem it{};
              it.src = stk;
              it.rows = p * k;
              it.ld = p * k;
              it.r_out = fin;
              it.ld_r = k;
              it.map = mo;
              it.leaf = b;
              it.k = k;
              tb_rows = std::max(tb_rows, it.rows);
              tb_stack.push_back(it);
            }
          }
          tb_k = std::max(tb_k, k);
          tb_core.push_back(c);
          continue;
        }
        const int q = K == 8 ? 0 : (K == 16 ? 1 : (K == 24 ? 2 : 3));
        const RkLeafDesc& d = desc[b];
        TsCore c{};
        c.leaf = b;
        c.k = h_ranks[b];
        for (int side = 0; side < 2; ++side) {
          const int len = side ? d.n : d.m;
          const long long base = d.ws_off + (side ? (long long)d.m * d.kcap : 0);
          const long long fin = tri_n, mo = map_n;
          tri_n += (long long)K * K;
          map_n += (long long)K * K;
          (side ? c.rb : c.ra) = fin;
          (side ? c.mb : c.ma) = mo;
          const int p = (len + kTsSegRows - 1) / kTsSegRows;
          long long stk = 0;
          if (p > 1) {
            stk = tri_n;
            tri_n += (long long)p * K * K;
          }
          for (int sg = 0; sg < p; ++sg) {
            TsItem it{};
            it.src = base + (long long)sg * kTsSegRows;
            it.rows = std::min(kTsSegRows, len - sg * kTsSegRows);
            it.ld = len;
            it.r_out = p == 1 ? fin : stk + (long long)sg * K;
            it.ld_r = p == 1 ? K : p * K;
            it.map = mo;
            it.leaf = b;
            it.k = c.k;
            ts_seg[q].push_back(it);
          }
          if (p > 1) {
            TsItem it{};
            it.src = stk;
            it.rows = p * K;
            it.ld = p * K;
            it.r_out = fin;
            it.ld_r = K;
            it.map = mo;
            it.leaf = b;
            it.k = c.k;
            ts_stack[q].push_back(it);
          }
        }
        ts_core[q].push_back(c);
        any_ts = true;
      }
      for (int b : good)
        if (jobs[b].svd) svd_good.push_back(b);
      if (!svd_good.empty()) {
        big_m = max_m;
        big_n = max_n;
        big_k = max_k;
      }
      if (!large.empty() || !svd_good.empty()) {
        slab = truncate_slab_elems<T>(big_m, big_n, big_k);
        // the slabs are sized for the largest leaf: let them use a third of the free memory
        // when that is more than the ACA budget, so long high-rank leaves still fill the grid
        size_t budget = workspace_budget();
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) budget = std::max(budget, free_b / 3);
        grid = std::min<long long>((long long)std::max(large.size(), svd_good.size()), persistent_grid(2));
        grid = std::max(1LL, std::min<long long>(grid, (long long)(budget / (slab * sizeof(W)))));
        d_scratch.alloc((size_t)(grid * slab));
      }
      if (any_ts) {
        d_tri.alloc((size_t)tri_n);
        d_maps.alloc((size_t)map_n);
        for (int q = 0; q < 4; ++q) {
          // longest segments first: the warps take items in order
          std::stable_sort(ts_seg[q].begin(), ts_seg[q].end(),
                           [](const TsItem& x, const TsItem& y) { return x.rows > y.rows; });
          std::stable_sort(ts_stack[q].begin(), ts_stack[q].end(),
                           [](const TsItem& x, const TsItem& y) { return x.rows > y.rows; });
          d_ts_seg[q].upload(ts_seg[q], stream_);
          d_ts_stack[q].upload(ts_stack[q], stream_);
          d_ts_core[q].upload(ts_core[q], stream_);
        }
      }
      if (!tb_core.empty()) {
        // slab a CTA: a segment (rows x k) with tau and R, or the core's two k x k blocks
        tb_slab = (long long)tb_rows * tb_k + tb_k + 3LL * tb_k * tb_k + 2LL * tb_k + 64;
        size_t budget = workspace_budget();
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) budget = std::max(budget, free_b / 3);
        long long g = std::min<long long>((long long)tb_seg.size(), persistent_grid(4));
        g = std::max(1LL, std::min<long long>(g, (long long)(budget / (tb_slab * sizeof(W)))));
        tb_grid = (int)g;
        d_tb_scratch.alloc((size_t)(g * tb_slab));
        d_tb_tri.alloc((size_t)tb_tri);
        d_tb_maps.alloc((size_t)tb_map);
        std::stable_sort(tb_seg.begin(), tb_seg.end(), [](const TsItem& x, const TsItem& y) { return x.rows > y.rows; });
        std::stable_sort(tb_stack.begin(), tb_stack.end(),
                         [](const TsItem& x, const TsItem& y) { return x.rows > y.rows; });
        d_tb_seg.upload(tb_seg, stream_);
        d_tb_stack.upload(tb_stack, stream_);
        d_tb_core.upload(tb_core, stream_);
      }
      d_svd_good.upload(svd_good, stream_);
      d_good.upload(large, stream_);
      HB_CUDA(cudaStreamSynchronize(stream_));
    }
    HB_CUDA(cudaEventRecord(ev_[4], stream_));
    if (!good.empty()) {
      if (!svd_good.empty()) {
        // SVD of the dense blocks at the compression epsilon (a stratum's dense sum: at the
        // low-rank epsilon, truncatedSvd in formattedAddParts), then the regular truncation
        HB_CUDA(cudaMemsetAsync(d_counter.p, 0, sizeof(int), stream_));
        launch_truncate<T>(d_desc.p, d_svd_good.p, (int)svd_good.size(), add_stratum ? eps_trunc : eps_aca, d_ws.p,
                           d_ranks.p, d_status.p,
                           d_counter.p, d_scratch.p, slab, (int)grid, stream_);
        HB_CUDA(cudaGetLastError());
      }
      // the tall-skinny phases hold leaves disjoint from the CTA kernel's: they run on a
      // second stream beside it
      if (any_ts) {
        HB_CUDA(cudaEventRecord(fork_[0], stream_));
        HB_CUDA(cudaStreamWaitEvent(stream2_, fork_[0], 0));
        for (int q = 0; q < 4; ++q) {
          const int K = 8 * (q + 1);
          launch_tsqr<T>(K, d_ts_seg[q].p, (int)ts_seg[q].size(), d_ws.p, d_tri.p, false, stream2_);
          launch_tsqr<T>(K, d_ts_stack[q].p, (int)ts_stack[q].size(), d_ws.p, d_tri.p, true, stream2_);
          launch_tscore<T>(K, d_ts_core[q].p, (int)ts_core[q].size(), d_tri.p, d_maps.p, d_ranks.p, d_status.p,
                           eps_trunc, stream2_);
          launch_tsapply<T>(K, d_ts_seg[q].p, (int)ts_seg[q].size(), d_ws.p, d_maps.p, d_ranks.p, stream2_);
          HB_CUDA(cudaGetLastError());
        }
        HB_CUDA(cudaEventRecord(fork_[1], stream2_));
      }
      if (!large.empty()) {
        HB_CUDA(cudaMemsetAsync(d_counter.p, 0, sizeof(int), stream_));
        launch_truncate<T>(d_desc.p, d_good.p, (int)large.size(), eps_trunc, d_ws.p, d_ranks.p, d_status.p,
                           d_counter.p, d_scratch.p, slab, (int)grid, stream_);
        HB_CUDA(cudaGetLastError());
      }
      if (!tb_core.empty()) {
        launch_tsqr_cta<T>(d_tb_seg.p, (int)tb_seg.size(), d_ws.p, d_tb_tri.p, false, d_tb_scratch.p, tb_slab,
                           tb_grid, d_counter.p, stream_);
        launch_tsqr_cta<T>(d_tb_stack.p, (int)tb_stack.size(), d_ws.p, d_tb_tri.p, true, d_tb_scratch.p, tb_slab,
                           tb_grid, d_counter.p, stream_);
        launch_tscore_cta<T>(d_tb_core.p, (int)tb_core.size(), d_tb_tri.p, d_tb_maps.p, d_ranks.p, d_status.p,
                             eps_trunc, d_tb_scratch.p, tb_slab, tb_grid, d_counter.p, stream_);
        launch_tsapply_cta<T>(d_tb_seg.p, (int)tb_seg.size(), d_ws.p, d_tb_maps.p, d_ranks.p, d_tb_scratch.p, tb_slab,
                              tb_grid, d_counter.p, stream_);
        HB_CUDA(cudaGetLastError());
      }
      if (any_ts) HB_CUDA(cudaStreamWaitEvent(stream_, fork_[1], 0));
    }
    HB_CUDA(cudaEventRecord(ev_[5], stream_));
    HB_CUDA(cudaMemcpyAsync(h_ranks.data(), d_ranks.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    HB_CUDA(cudaMemcpyAsync(h_status.data(), d_status.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    HB_CUDA(cudaStreamSynchronize(stream_));
    HB_CUDA(cudaEventElapsedTime(&ms, ev_[4], ev_[5]));
    times_ms[2] += ms;
    for (int b = 0; b < nb; ++b) {
      if (h_status[b] == kLeafAcaCapacity) h_ranks[b] = 0;
      else if (h_status[b] != kLeafOk)
        throw Error("truncation failed on leaf " + std::to_string(jobs[b].leaf) +
                    (h_status[b] == kLeafSvdNoConverge
                         ? ": the Jacobi SVD of its core did not converge within " + std::to_string(jacobi_sweeps()) +
                               " sweeps"
                         : " (status " + std::to_string(h_status[b]) + ")"));
    }
    // storage of each leaf in the new piece: A row panels, then B^T
    std::vector<RkStoreDesc> store(nb);
    std::vector<PanelDesc> panels;
    std::vector<long long> loff(nb, -1);
    long long pe = 0;
    for (int b = 0; b < nb; ++b) {
      store[b] = RkStoreDesc{(int)panels.size(), 0, 0};
      const int k = h_ranks[b];
      if (k <= 0) continue;
      const LeafInfo& l = L[jobs[b].leaf];
      loff[b] = pe;
      auto br = block_range(rblocks_, rstarts_, l.row_off, l.m);
      for (int q = br.first; q < br.second; ++q) {
        panels.push_back(PanelDesc{rblocks_[q].off - l.row_off, rblocks_[q].len, pe});
        pe += padded((long long)rblocks_[q].len * k);
        store[b].npanel++;
      }
      store[b].bt_off = pe;
      pe += padded((long long)k * l.n);
    }
    HB_CUDA(cudaMemcpyAsync(d_ranks.p, h_ranks.data(), nb * sizeof(int), cudaMemcpyHostToDevice, stream_));
    Piece piece;
    piece.arena.alloc((size_t)std::max(pe, 1LL) + 64);
    piece.elems = pe;
    DevArray<RkStoreDesc> d_store;
    DevArray<PanelDesc> d_panels;
    d_store.upload(store, stream_);
    d_panels.upload(panels, stream_);
    HB_CUDA(cudaEventRecord(ev_[4], stream_));
    launch_compact<T>(d_desc.p, nb, d_ws.p, d_ranks.p, d_store.p, d_panels.p, piece.arena.p, stream_);
    HB_CUDA(cudaGetLastError());
    HB_CUDA(cudaEventRecord(ev_[5], stream_));
    HB_CUDA(cudaStreamSynchronize(stream_));
    HB_CUDA(cudaEventElapsedTime(&ms, ev_[4], ev_[5]));
    times_ms[2] += ms;
    const int pid = (int)pieces_.size();
    for (int b = 0; b < nb; ++b) {
      if (h_status[b] == kLeafAcaCapacity) continue;
      const int leaf = jobs[b].leaf;
      ranks[leaf] = h_ranks[b];
      piece_of_[leaf] = h_ranks[b] > 0 ? pid : -1;
      piece_loff_[leaf] = loff[b];
    }
    pieces_.push_back(std::move(piece));
  }

  void assemble_rk(int method, double eps_aca, double eps_trunc, int svd_below, int stratum) {
    HB_CUDA(set_jacobi_max_sweeps(jacobi_sweeps()));
    (void)method;
    const auto& L = bt_->leaves;
    const int nleaves = (int)L.size();
    piece_of_.assign(nleaves, -1);
    pieces_.clear();
    for (int bk = 0; bk < kAcaBuckets; ++bk) {
      aca_shape[bk] = -1;
      aca_tuned[bk] = 0;
      for (double& r : aca_rate[bk]) r = 0.0;
    }
    std::vector<RkJob> queue;
    const int k0 = initial_kcap();
    for (int i = 0; i < nleaves; ++i) {
      if (L[i].type != 1) continue;
      ranks[i] = 0;
      RkJob j;
      j.leaf = i;
      j.svd = std::max(L[i].m, L[i].n) < svd_below;
      const int mn = std::min(L[i].m, L[i].n);
      j.kcap = j.svd ? mn : std::min(mn, k0);
      queue.push_back(j);
    }
    const size_t budget = workspace_budget();
    while (!queue.empty()) {
      std::vector<RkJob> retry;
      size_t pos = 0;
      while (pos < queue.size()) {
        std::vector<RkJob> batch;
        size_t bytes = 0;
        while (pos < queue.size()) {
          const LeafInfo& l = L[queue[pos].leaf];
          size_t b = (size_t)pad32(rk_slot_elems(l.m, l.n, queue[pos].kcap)) * sizeof(T) + l.m + l.n;
          if (!batch.empty() && bytes + b > budget) break;
          bytes += b;
          batch.push_back(queue[pos++]);
        }
        run_batch(batch, eps_aca, eps_trunc, retry, nullptr, stratum);
      }
      queue.swap(retry);
    }
  }

  // The plain kernel of stratum s: the stratum's parameter, no nugget (its weight scales A).
  KernelParams stratum_kp(int s) const {
    KernelParams k = kp_;
    k.nstrata = 0;
    k.strata = nullptr;
    const double a = strata_[s];
    if (k.kind == kExpCov) {
      k.ell = a;
      k.nugget = 0.0;
    } else if (k.kind == kLaplaceReg) {
      k.delta = a;
    } else {
      k.wavenumber = a;
    }
    return k;
  }

  // Stratum s after its ACA in run_batch (h_ranks: the stratum's ranks).  Stratum 0: A scaled
  // by the stratum's weight, in place.  A further stratum: a new workspace whose slot b holds
  // the factors leaf b holds (kcur columns, unpacked from the arena) followed by the stratum's
  // (A scaled by its weight); a leaf whose summed rank reaches min(m, n) holds the exact
  // factorisation of its full block instead and becomes an SVD job; a leaf with no new column
  // keeps its factors and skips the truncation.  Leaves out of ACA capacity are left for the
  // retry (their slots hold nothing).
  void join_stratum(int s, std::vector<RkJob>& jobs, std::vector<RkLeafDesc>& desc, DevArray<RkLeafDesc>& d_desc,
                    DevArray<T>& d_ws, DevArray<int>& d_ranks, const std::vector<int>& h_status,
                    std::vector<int>& h_ranks, const T* src) {
    const int nb = (int)jobs.size();
    const double w = strata_[kp_.nstrata + s];
    if (s == 0) {
      if (w == 1.0) return;
      std::vector<int> list;
      for (int b = 0; b < nb; ++b)
        if (!jobs[b].svd && !jobs[b].pass && h_status[b] == kLeafOk && h_ranks[b] > 0) list.push_back(b);
      DevArray<int> d_list;
      d_list.upload(list, stream_);
      launch_scale_a<T>(d_desc.p, d_list.p, (int)list.size(), d_ranks.p, w, d_ws.p, stream_);
      HB_CUDA(cudaGetLastError());
      HB_CUDA(cudaStreamSynchronize(stream_));
      return;
    }
    std::vector<RkLeafDesc> desc2(desc);
    std::vector<int> kcur(nb, 0), ks(nb, 0), kcat(nb, 0), dense;
    std::vector<long long> dof;
    long long ws2 = 0, dsz = 0;
    for (int b = 0; b < nb; ++b) {
      const RkLeafDesc& d = desc[b];
      int cap = 1;
      if (h_status[b] == kLeafOk) {
        kcur[b] = jobs[b].kcur;
        ks[b] = jobs[b].pass ? 0 : h_ranks[b];
        kcat[b] = kcur[b] + ks[b];
        cap = std::max(1, kcat[b]);
        if (ks[b] > 0 && kcat[b] >= std::min(d.m, d.n)) {
          dense.push_back(b);
          dof.push_back(dsz);
          dsz += padded((long long)d.m * d.n);
        }
      }
      desc2[b].kcap = cap;
      desc2[b].ws_off = ws2;
      ws2 += pad32(rk_slot_elems(d.m, d.n, cap));
    }
    std::vector<RkStoreDesc> ostore(nb);
    std::vector<PanelDesc> opanels;
    for (int b = 0; b < nb; ++b)
      ostore[b] = kcur[b] > 0 ? rk_store(jobs[b].leaf, opanels) : RkStoreDesc{0, 0, 0, 0, 0};
    DevArray<RkLeafDesc> d_desc2;
    DevArray<T> ws_new;
    DevArray<RkStoreDesc> d_ostore;
    DevArray<PanelDesc> d_opanels;
    DevArray<int> d_kcur, d_ks, d_kcat, d_dense;
    DevArray<long long> d_dof;
    DevArray<T> scratch;
    d_desc2.upload(desc2, stream_);
    ws_new.alloc((size_t)std::max(ws2, 1LL));
    d_ostore.upload(ostore, stream_);
    d_opanels.upload(opanels, stream_);
    d_kcur.upload(kcur, stream_);
    d_ks.upload(ks, stream_);
    d_kcat.upload(kcat, stream_);
    d_dense.upload(dense, stream_);
    d_dof.upload(dof, stream_);
    launch_unpack<T>(d_desc2.p, nb, d_kcur.p, d_ostore.p, d_opanels.p, src, ws_new.p, stream_);
    launch_append_factors<T>(d_desc.p, d_desc2.p, nb, d_kcur.p, d_ks.p, w, d_ws.p, ws_new.p, stream_);
    if (!dense.empty()) {
      scratch.alloc((size_t)dsz);
      launch_exact_factors<T>(d_desc2.p, d_dense.p, (int)dense.size(), d_kcur.p, d_kcat.p, d_dof.p, ws_new.p,
                              scratch.p, stream_);
    }
    HB_CUDA(cudaGetLastError());
    for (int b = 0; b < nb; ++b) {
      if (h_status[b] != kLeafOk) continue;
      h_ranks[b] = kcat[b];
      if (ks[b] == 0) jobs[b].pass = true;  // nothing joined: kept as held
    }
    for (int b : dense) {
      h_ranks[b] = std::min(desc[b].m, desc[b].n);
      jobs[b].svd = true;
    }
    HB_CUDA(cudaMemcpyAsync(d_ranks.p, h_ranks.data(), nb * sizeof(int), cudaMemcpyHostToDevice, stream_));
    HB_CUDA(cudaStreamSynchronize(stream_));
    desc.swap(desc2);
    d_desc.swap(d_desc2);
    d_ws.swap(ws_new);
  }

  // Stratum s (>= 1) of a multi-strata kernel joined to the assembled leaves: every admissible
  // leaf compressed by ACA runs the stratum's ACA (capacity retries as in assemble_rk), the
  // dense-SVD leaves keep their factors (the SVD compression is not incremental:
  // compression.hpp:103), then the arena is rebuilt for the new ranks.
  void add_stratum(int s, double eps_aca, double eps_trunc) {
    const auto& L = bt_->leaves;
    const int nleaves = (int)L.size();
    const int k0 = initial_kcap();
    std::vector<RkJob> queue;
    for (int i = 0; i < nleaves; ++i) {
      if (L[i].type != 1) continue;
      RkJob j;
      j.leaf = i;
      j.svd = false;
      j.kcur = std::max(0, ranks[i]);
      if (std::max(L[i].m, L[i].n) < svd_below_) {
        if (j.kcur == 0) continue;
        j.pass = true;
        j.kcap = 1;
      } else {
        j.kcap = std::min(std::min(L[i].m, L[i].n), k0);
      }
      queue.push_back(j);
    }
    piece_of_.assign(nleaves, -1);
    piece_loff_.assign(nleaves, -1);
    pieces_.clear();
    const size_t budget = workspace_budget();
    while (!queue.empty()) {
      std::vector<RkJob> retry;
      size_t pos = 0;
      while (pos < queue.size()) {
        std::vector<RkJob> batch;
        size_t bytes = 0;
        while (pos < queue.size()) {
          const RkJob& j = queue[pos];
          const LeafInfo& l = L[j.leaf];
          // the stratum's ACA slot and the joined slot
          size_t b = (size_t)(pad32(rk_slot_elems(l.m, l.n, j.kcap)) + pad32(rk_slot_elems(l.m, l.n, j.kcur + j.kcap))) *
                         sizeof(T) + l.m + l.n;
          if (!batch.empty() && bytes + b > budget) break;
          bytes += b;
          batch.push_back(queue[pos++]);
        }
        run_batch(batch, eps_aca, eps_trunc, retry, arena_.p, s);
      }
      queue.swap(retry);
    }
    float ms = 0;
    rebuild_arena(&ms);
    times_ms[0] += ms;
  }

  // A new arena for new ranks: the full leaves' panels moved from the current one, the Rk
  // factors from their pieces (with `timed`, the device time of the placement added to it).
  void rebuild_arena(float* timed = nullptr) {
    const auto& L = bt_->leaves;
    const int nleaves = (int)L.size();
    const Layout old = layout_;
    compute_layout();
    DevArray<T> na;
    na.alloc((size_t)(layout_.total + 256));
    HB_CUDA(cudaMemsetAsync(na.p, 0, (size_t)layout_.total * sizeof(T), stream_));
    std::vector<CopySeg> segs;
    for (int i = 0; i < nleaves; ++i) {
      if (L[i].type != 0 || layout_.first[i] < 0) continue;
      auto br = block_range(rblocks_, rstarts_, L[i].row_off, L[i].m);
      for (int b = br.first; b < br.second; ++b)
        segs.push_back(CopySeg{old.panel[old.first[i] + (b - br.first)], layout_.panel[layout_.first[i] + (b - br.first)],
                               rblocks_[b].len * L[i].n, 1, 0, 0});
    }
    DevArray<CopySeg> d_segs;
    d_segs.upload(segs, stream_);
    launch_copy_segments<T>(d_segs.p, (int)segs.size(), arena_.p, na.p, stream_);
    HB_CUDA(cudaGetLastError());
    scatter_pieces(na.p, timed);
    arena_.swap(na);
    pieces_.clear();
  }

  // ------------------------------------------------------------------------------
  // Arena layout.  Region Y: per output block b (rblocks_, O_b rows), the row panels of every
  // leaf whose rows cover b, side by side in leaf order as one column-major O_b x W_b matrix
  // (a full leaf's panel has n columns, an Rk leaf's A panel k columns), W_b rounded up to a
  // multiple of kYColAlign with zero columns; so a leaf's panel for b is still one contiguous
  // O_b x w chunk.  Region BT: per Rk leaf of rank k > 0, B^T (k x n, column-major), 16-byte
  // aligned.  The 'N' product streams each block's matrix in one pass; every piece of it and
  // every B^T starts on a 16-byte boundary (the TMA rule).
  // A group of Rk leaves with one column range: their B^T stacked as one column-major h x n
  // matrix (leaf order, at most kZGroupRows rows unless one leaf has more), so that one pass
  // over its columns computes the z = B^T x of all of them with the x rows read once.
  struct ZGroup {
    long long base;
    int h, col_off, n;
    std::vector<int> leaves;  // member leaves, rows in this order
  };
  static constexpr int kZGroupRows = 32;
  struct Layout {
    std::vector<int> first;         // per leaf: its first entry in `panel`, -1 without storage
    std::vector<long long> panel;   // per (leaf, block of its rows): offset of the leaf's panel
    std::vector<int> pcol;          // its first column in the block's matrix
    std::vector<long long> bt;      // per leaf: offset of B^T, -1 unless Rk with rank > 0
    std::vector<int> bt_ld;         // per leaf: leading dimension of B^T (its group's height)
    std::vector<long long> yblock;  // per output block: offset of its matrix
    std::vector<int> ywidth;        // per output block: columns (a multiple of kYColAlign)
    std::vector<ZGroup> zgroups;    // the B^T groups, in the region's order
    long long total = 0;
  };

  bool has_storage(int i) const {
    const LeafInfo& l = bt_->leaves[i];
    if (l.m == 0 || l.n == 0) return false;
    return l.type == 0 || ranks[i] > 0;
  }

  void compute_layout() {
    const auto& L = bt_->leaves;
    const int nleaves = (int)L.size();
    Layout y;
    y.first.assign(nleaves, -1);
    y.bt.assign(nleaves, -1);
    std::vector<int> width(rblocks_.size(), 0);
    for (int i = 0; i < nleaves; ++i) {
      if (!has_storage(i)) continue;
      const int w = L[i].type == 0 ? L[i].n : ranks[i];
      auto br = block_range(rblocks_, rstarts_, L[i].row_off, L[i].m);
      y.first[i] = (int)y.pcol.size();
      for (int b = br.first; b < br.second; ++b) {
        y.pcol.push_back(width[b]);
        width[b] += w;
      }
    }
    long long pos = 0;
    y.yblock.resize(rblocks_.size());
    y.ywidth.resize(rblocks_.size());
    for (size_t b = 0; b < rblocks_.size(); ++b) {
      y.yblock[b] = pos;
      y.ywidth[b] = (width[b] + kYColAlign - 1) / kYColAlign * kYColAlign;
      pos += (long long)rblocks_[b].len * y.ywidth[b];
    }
    y.panel.resize(y.pcol.size());
    for (int i = 0; i < nleaves; ++i) {
      if (y.first[i] < 0) continue;
      auto br = block_range(rblocks_, rstarts_, L[i].row_off, L[i].m);
      for (int b = br.first; b < br.second; ++b) {
        const int e = y.first[i] + (b - br.first);
        y.panel[e] = y.yblock[b] + (long long)y.pcol[e] * rblocks_[b].len;
      }
    }
    // Region BT: Rk leaves with the same column range (in order of first appearance) stacked
    // in groups of at most kZGroupRows rows
    pos = pad32(pos);
    y.bt_ld.assign(nleaves, 0);
    std::map<std::pair<int, int>, int> by_cols;
    std::vector<std::vector<int>> members;
    for (int i = 0; i < nleaves; ++i) {
      if (L[i].type != 1 || y.first[i] < 0) continue;
      auto key = std::make_pair(L[i].col_off, L[i].n);
      auto it = by_cols.find(key);
      if (it == by_cols.end()) {
        it = by_cols.emplace(key, (int)members.size()).first;
        members.emplace_back();
      }
      members[it->second].push_back(i);
    }
    for (const auto& mem : members) {
      ZGroup g{0, 0, L[mem[0]].col_off, L[mem[0]].n, {}};
      auto close = [&]() {
        if (g.leaves.empty()) return;
        g.base = pos;
        int r = 0;
        for (int i : g.leaves) {
          y.bt[i] = pos + r;
          y.bt_ld[i] = g.h;
          r += ranks[i];
        }
        pos += padded((long long)g.h * g.n);
        y.zgroups.push_back(g);
        g.leaves.clear();
        g.h = 0;
      };
      for (int i : mem) {
        if (g.h > 0 && g.h + ranks[i] > kZGroupRows) close();
        g.leaves.push_back(i);
        g.h += ranks[i];
      }
      close();
    }
    y.total = pad32(pos);
    layout_ = std::move(y);
  }

  // Descriptors of the full leaves' row panels in the current layout (and, with `goff`, their
  // canonical offsets).
  void full_descs(std::vector<FullLeafDesc>& fd, std::vector<PanelDesc>& fp, std::vector<long long>* fgoff,
                  const std::vector<long long>* goff = nullptr) const {
    const auto& L = bt_->leaves;
    for (int i = 0; i < (int)L.size(); ++i) {
      if (L[i].type != 0 || layout_.first[i] < 0) continue;
      FullLeafDesc d{L[i].row_off, L[i].m, L[i].col_off, L[i].n, (int)fp.size(), 0};
      auto br = block_range(rblocks_, rstarts_, L[i].row_off, L[i].m);
      for (int b = br.first; b < br.second; ++b) {
        fp.push_back(PanelDesc{rblocks_[b].off - L[i].row_off, rblocks_[b].len,
                               layout_.panel[layout_.first[i] + (b - br.first)]});
        d.npanel++;
      }
      fd.push_back(d);
      if (fgoff) fgoff->push_back((*goff)[i]);
    }
  }

  // Where Rk leaf i's factors live in the current layout: its A panels appended to `panels`.
  RkStoreDesc rk_store(int i, std::vector<PanelDesc>& panels) const {
    const LeafInfo& l = bt_->leaves[i];
    RkStoreDesc st{(int)panels.size(), 0, layout_.bt[i], layout_.first[i] < 0 ? 0 : layout_.bt_ld[i], 0};
    if (layout_.first[i] < 0) return st;
    auto br = block_range(rblocks_, rstarts_, l.row_off, l.m);
    for (int b = br.first; b < br.second; ++b) {
      panels.push_back(PanelDesc{rblocks_[b].off - l.row_off, rblocks_[b].len,
                                 layout_.panel[layout_.first[i] + (b - br.first)]});
      st.npanel++;
    }
    return st;
  }

  // The compacted factors of every piece (A row panels, then B^T, per leaf at piece_loff_)
  // into their places in `dst` (laid out by layout_).
  // With `timed`, the device time of the copies is added to *timed (ms).
  void scatter_pieces(T* dst, float* timed = nullptr) {
    const auto& L = bt_->leaves;
    std::vector<std::vector<CopySeg>> segs(pieces_.size());
    for (int i = 0; i < (int)L.size(); ++i) {
      if (L[i].type != 1 || piece_of_[i] < 0 || layout_.first[i] < 0) continue;
      const int k = ranks[i];
      auto br = block_range(rblocks_, rstarts_, L[i].row_off, L[i].m);
      long long p = piece_loff_[i];
      for (int b = br.first; b < br.second; ++b) {
        const int len = rblocks_[b].len * k;
        segs[piece_of_[i]].push_back(CopySeg{p, layout_.panel[layout_.first[i] + (b - br.first)], len, 1, 0, 0});
        p += padded(len);
      }
      // B^T: k x n in the piece, rows of its group's matrix in the arena
      segs[piece_of_[i]].push_back(CopySeg{p, layout_.bt[i], k, L[i].n, k, layout_.bt_ld[i]});
    }
    std::vector<DevArray<CopySeg>> d_segs(pieces_.size());
    for (size_t q = 0; q < pieces_.size(); ++q) d_segs[q].upload(segs[q], stream_);
    if (timed) HB_CUDA(cudaEventRecord(ev_[2], stream_));
    for (size_t q = 0; q < pieces_.size(); ++q) {
      launch_copy_segments<T>(d_segs[q].p, (int)segs[q].size(), pieces_[q].arena.p, dst, stream_);
      HB_CUDA(cudaGetLastError());
    }
    if (timed) HB_CUDA(cudaEventRecord(ev_[3], stream_));
    HB_CUDA(cudaStreamSynchronize(stream_));
    if (timed) {
      float ms = 0;
      HB_CUDA(cudaEventElapsedTime(&ms, ev_[2], ev_[3]));
      *timed += ms;
    }
  }

  // ------------------------------------------------------------------------------
  // gemv schedule
  struct SideBuf {
    DevArray<GemvUnit> units;
    DevArray<GemvTask> tasks[GemvSide::kMaxLaunch + 1];
    DevArray<int> begin[GemvSide::kMaxLaunch + 1];
    DevArray<GemvZred> zred;
    DevArray<int> zcnt;
    DevArray<int2> yrows;
  };

  // Whether the z kernels sum the chunks of long groups themselves (the warp finishing a sum's
  // last chunk adds the parts) instead of a separate pass: the 'N' products in FP64 and complex
  // (cylinder 100,000, 16 RHS, FP64: z-phase 0.385 -> 0.352 ms).  Not the FP32 tensor-core
  // z-phase, whose short kernel ends later by the chunks' fences and the last warps' sums than
  // the separate pass takes (0.134 -> 0.141 ms).
  static bool zsum_in_kernel(bool trans) { return !trans && !kTensorN; }

  static int rank_class(int k) { return k <= 16 ? 0 : (k <= 32 ? 1 : (k <= 64 ? 2 : 3)); }
  static void class_shape(int c, int& ol, int& rpt) {
    ol = c == 0 ? 16 : 32;
    rpt = c <= 1 ? 1 : (c == 2 ? 2 : 4);
  }

  // Columns per unit of a warp-level launch: the piece (O x cols) and its X rows fit one
  // pipeline stage at the widest right-hand-side tile.
  static int warp_unit_cols(int O) {
    const int Rmax = sizeof(T) >= 16 ? 4 : 16;
    const int xrow_bytes = gemv_rhs_stride((int)sizeof(T), Rmax) * (int)sizeof(T);
    // pieces start 16-byte aligned when cols * O * sizeof(T) is a multiple of 16
    const int g = sizeof(T) >= 16 ? 1 : 16 / (int)sizeof(T);
    int cols = std::min(kWarpXBytes / xrow_bytes, warp_piece_bytes((int)sizeof(T)) / (O * (int)sizeof(T)));
    cols -= cols % g;
    if (cols < g) throw Error("gemv plan: output too tall for a warp-level unit");
    return cols;
  }
  // Columns and X offset of the units of a piece of O rows.  FP32: the stage split the other
  // way (kWarpXBytesWide of X rows) when that gives wider units, as for B^T blocks of ranks
  // below 16 (40 columns at rank 12 instead of 32).  Other types: the widest aligned unit whose
  // piece and X rows fit the stage together, the X rows right after the piece (16-byte
  // aligned), instead of the fixed split whose X part held 16 FP64 rows whatever O: the FP64
  // z-phase units of a rank-12 group take 30 columns instead of 16, the y-phase's 64-row
  // blocks 10 instead of 8.
  static int warp_unit_cols_wide(int O, int* xoff) {
    const int cols = warp_unit_cols(O);
    *xoff = warp_piece_bytes((int)sizeof(T));
    if (!std::is_same<T, float>::value) {
      const int s = (int)sizeof(T);
      const int Rmax = s >= 16 ? 4 : 16;
      const long long xrow = (long long)gemv_rhs_stride(s, Rmax) * s;
      const int g = s >= 16 ? 1 : 16 / s;  // the next piece starts 16-byte aligned
      const long long stage = warp_piece_bytes(s) + kWarpXBytes;
      auto need = [&](long long c) { return ((long long)O * c * s + 15) / 16 * 16 + c * xrow; };
      long long c = cols;
      while (need(c + g) <= stage) c += g;
      if (need(c) > stage) throw Error("gemv plan: output too tall for a warp-level unit");
      *xoff = (int)(((long long)O * c * s + 15) / 16 * 16);
      return (int)c;
    }
    const int stage = warp_piece_bytes(4) + kWarpXBytes;
    const int xrow_bytes = gemv_rhs_stride(4, 16) * 4;
    int wide = std::min(kWarpXBytesWide / xrow_bytes, (stage - kWarpXBytesWide) / (O * 4));
    wide -= wide % 4;
    if (wide <= cols) return cols;
    *xoff = stage - kWarpXBytesWide;
    return wide;
  }

  // Tensor-core units (FP32, FP64): the widest multiple of the kernel's column step (8 for the
  // TF32 MMA, 4 for the FP64 one) whose piece (O x c) and X rows (c rows of 16 scalars) fit
  // one pipeline stage, the X rows right after the piece (16-byte aligned); *xoff is their
  // offset in the stage.
  static int mma_unit_cols(int O, int* xoff) {
    const int s = (int)sizeof(T);
    const int stage = warp_piece_bytes(s) + kWarpXBytes;
    const int xrow = gemv_rhs_stride(s, 16) * s;
    const int step = s == 4 ? 8 : 4;
    auto need = [&](int c) { return (((long long)O * c * s + 15) / 16) * 16 + (long long)c * xrow; };
    int c = step;
    while (need(c + step) <= stage) c += step;
    if (need(c) > stage) throw Error("gemv plan: output too tall for a tensor-core unit");
    *xoff = (int)(((long long)O * c * s + 15) / 16 * 16);
    return c;
  }
  static constexpr bool kTensorN = std::is_same<T, float>::value;  // 'N' products on the TF32 tensor-core kernel

  // Units of out(O rows) += P X for a column-major O x C block at `poff`, X rows from `xrow`,
  // `cols` columns per unit.
  void px_units(std::vector<GemvUnit>& u, long long poff, int O, int C, int xrow, int cols = 32,
                int xoff = warp_piece_bytes((int)sizeof(T))) {
    for (int j0 = 0; j0 < C; j0 += cols) {
      GemvUnit g{};  // nruns = 0: contiguous X rows
      g.poff = poff + (long long)j0 * O;
      g.xrow = xrow + j0;
      g.c = std::min(cols, C - j0);
      g.o0 = xoff;  // X rows' offset in a warp-level stage
      g.ow = O;
      g.pel = O * g.c;
      g.shift = (int)(g.poff % kPad);
      if (g.shift) throw Error("gemv plan: misaligned panel piece");
      u.push_back(g);
    }
  }
  // Units of out[o_base + w] += sum_i P[i, w] X[i] for a column-major C x W block at `poff`.
  void ptx_units(std::vector<GemvUnit>& u, long long poff, int C, int W, int o_base, int xrow) {
    if (C > 128) throw Error("gemv plan: transposed inner extent above 128 (rank or block too large)");
    for (int w0 = 0; w0 < W; w0 += 32) {
      GemvUnit g{};  // nruns = 0: contiguous X rows
      g.poff = poff + (long long)w0 * C;
      g.xrow = xrow;
      g.c = C;
      g.o0 = o_base + w0;
      g.ow = std::min(32, W - w0);
      g.pel = C * g.ow;
      g.shift = (int)(g.poff % kPad);
      u.push_back(g);
    }
  }

  // Contiguous ranges of tasks of about equal bytes for a persistent grid: one range per
  // CTA, or per warp for warp-level launches.  Returns the range starts; *ncta is the grid.
  // CTAs of the persistent grid of a launch: as many as fit the SMs at once.
  static int launch_ctas(int omax, bool transposed, bool warp_level, int map) {
    const int Rmax = sizeof(T) >= 16 ? 4 : 16;
    const int RS16 = gemv_rhs_stride((int)sizeof(T), Rmax);
    const size_t smem = map == 4      ? umma_smem_bytes()
                        : warp_level ? warp_stream_smem_bytes((int)sizeof(T))
                                     : stream_smem_bytes((int)sizeof(T), Rmax, RS16, omax, transposed);
    // warp-level kernels: 228 KB of shared memory an SM, 1 KB reserved a CTA (their launch
    // bounds guarantee the registers for that many CTAs)
    // (shared memory is allocated in 128-byte granules)
    const size_t alloc = (smem + 127) / 128 * 128;
    int per_sm = (int)std::min<size_t>(8, ((warp_level ? 228 : 226) * 1024) / (alloc + 1024));
    if (map == 3) per_sm = std::min(per_sm, mma_stream_blocks_per_sm(omax / 8, (int)sizeof(T)));  // registers
    per_sm = std::max(per_sm, 1);
    return persistent_grid(per_sm);
  }

  std::vector<int> partition(const std::vector<GemvTask>& tasks, const std::vector<GemvUnit>& units, int omax,
                             bool transposed, bool warp_level, int map, int* ncta) {
    const int Rmax = sizeof(T) >= 16 ? 4 : 16;
    const int RS16 = gemv_rhs_stride((int)sizeof(T), Rmax);
    const int wpc = warp_level ? warp_stream_warps_per_cta() : 1;
    const int nt = (int)tasks.size();
    const int cta = std::max(1, std::min((nt + wpc - 1) / wpc, launch_ctas(omax, transposed, warp_level, map)));
    *ncta = cta;
    const int G = cta * wpc;
    std::vector<double> cost(tasks.size());
    double tot = 0;
    for (size_t t = 0; t < tasks.size(); ++t) {
      double c = 0;
      for (int u = tasks[t].first_unit; u < tasks[t].first_unit + tasks[t].nunits; ++u)
        c += (double)units[u].pel + (double)units[u].c * RS16 + 64;
      cost[t] = c;
      tot += c;
    }
    std::vector<int> begin(G + 1, (int)tasks.size());
    begin[0] = 0;
    double acc = 0;
    int g = 1;
    for (size_t t = 0; t < tasks.size() && g < G; ++t) {
      acc += cost[t];
      while (g < G && acc >= tot * g / G) begin[g++] = (int)t + 1;
    }
    for (; g < G; ++g) begin[g] = (int)tasks.size();
    begin[G] = (int)tasks.size();
    return begin;
  }

  // Warp-level shape of an 'N' launch for tasks of at most omax rows: the column-slice
  // window (2 rows per lane) up to 32 rows, half-warp row groups up to 64, lanes over rows
  // up to 128 (4 rows per lane).
  static void warp_shape(GemvLaunch& L, int omax) {
    L.warp_level = true;
    L.ol = 32;
    if (std::is_same<T, float>::value) {
      // FP32: tensor-core tiles of 8 output rows (map 3, rpt = row tiles held per warp: exactly
      // those of the tallest task up to 8, else 16)
      L.map = 3;
      const int tiles = (omax + 7) / 8;
      L.rpt = tiles <= 8 ? tiles : 16;
      return;
    }
    // up to 32 rows: column-slice windows, 2 rows a lane; up to 64: lanes over rows, 2 rows a
    // lane (map 5: half the accumulators of the half-warp map 1, so twice the resident warps
    // with 16 FP64 right-hand sides); above: lanes over rows, 4 rows a lane
    L.map = omax <= 32 ? 2 : (omax <= 64 ? (gemv_half_warp_map() ? 1 : 5) : 0);
    L.rpt = omax <= 32 ? 2 : 4;
  }

  // With `begin` given (one range of tasks per warp, or per CTA, of the full persistent grid),
  // the ranges are taken as they are instead of being cut by cost here.
  void finish_launch(GemvLaunch& L, SideBuf& sb, int slot, std::vector<GemvTask>& tasks,
                     const std::vector<GemvUnit>& units, int ol, int rpt, bool transposed, bool out_is_y,
                     const std::vector<int>* begin_given = nullptr) {
    L.ntasks = (int)tasks.size();
    if (!L.warp_level) {
      L.ol = ol;
      L.rpt = rpt;
    }
    L.transposed = transposed;
    L.out_is_y = out_is_y;
    if (tasks.empty()) return;
    // X rows of every unit: contiguous, or at most kUnitRuns runs covering exactly c rows
    for (auto& t : tasks)
      for (int u = t.first_unit; u < t.first_unit + t.nunits; ++u) {
        const GemvUnit& g = units[u];
        if (g.nruns < 0 || g.nruns > kUnitRuns) throw Error("gemv plan: unit with a bad run count");
        if (g.nruns > 0) {
          long long rows = 0;
          for (int r = 0; r < g.nruns; ++r) rows += g.run_len[r];
          if (rows != g.c) throw Error("gemv plan: unit runs do not cover its columns");
          if (transposed) throw Error("gemv plan: runs of X rows in a transposed unit");  // read as one block
        }
      }
    // the kernel walks units sequentially across the tasks of a CTA
    for (size_t t = 1; t < tasks.size(); ++t)
      if (tasks[t].first_unit != tasks[t - 1].first_unit + tasks[t - 1].nunits)
        throw Error("gemv plan: units of a launch are not contiguous");
    const int omax = L.map == 4       ? 128
                     : L.warp_level ? (L.map == 3 ? 8 * L.rpt : (L.map == 2 ? 32 : (L.map == 1 || L.map == 5 ? 64 : 128)))
                                    : ol * rpt;
    for (auto& t : tasks)
      if (t.O > omax) throw Error("gemv plan: task taller than its launch shape");
    if (L.warp_level) {
      // every unit of the launch must fit one stage of the per-warp pipeline
      const int Rmax = sizeof(T) >= 16 ? 4 : 16;
      const long long xrow_bytes = (long long)gemv_rhs_stride((int)sizeof(T), Rmax) * sizeof(T);
      for (auto& t : tasks)
        for (int u = t.first_unit; u < t.first_unit + t.nunits; ++u) {
          const GemvUnit& g = units[u];
          // every unit carries its stage split: the X rows at byte o0, after the piece
          const long long stage = warp_piece_bytes((int)sizeof(T)) + kWarpXBytes;
          const long long xoff = g.o0;
          if (xoff % 16 != 0 || xoff <= 0 || xoff > stage || (long long)g.pel * sizeof(T) > xoff || g.shift != 0 ||
              g.c * xrow_bytes > stage - xoff)
            throw Error("gemv plan: unit above the warp-level stage capacity");
        }
    }
    if (L.map == 4) {
      // every unit must fit one stage of the tensor-memory kernel
      for (auto& t : tasks)
        for (int u = t.first_unit; u < t.first_unit + t.nunits; ++u) {
          const GemvUnit& g = units[u];
          if ((long long)g.pel * 4 > kTcPieceBytes || g.c > kTcCols || g.shift != 0 || g.c * 16 * 4 > kTcXBytes)
            throw Error("gemv plan: unit above the tensor-memory stage capacity");
        }
    }
    std::vector<int> begin;
    if (begin_given) {
      const int wpc = L.warp_level ? warp_stream_warps_per_cta() : 1;
      L.ncta = launch_ctas(omax, transposed, L.warp_level, L.map);
      begin = *begin_given;
      if ((int)begin.size() != L.ncta * wpc + 1 || begin.front() != 0 || begin.back() != (int)tasks.size())
        throw Error("gemv plan: task ranges do not match the launch grid");
    } else {
      begin = partition(tasks, units, omax, transposed, L.warp_level, L.map, &L.ncta);
    }
    sb.tasks[slot].upload(tasks, stream_);
    sb.begin[slot].upload(begin, stream_);
    L.tasks = sb.tasks[slot].p;
    L.cta_begin = sb.begin[slot].p;
  }

  // Builds one side: 'N' (trans = false) or 'T' / 'C'.
  void build_side(bool trans, const std::vector<GemvRkLeaf>& K, const std::vector<int>& rk_leaf,
                  long long& next_row, GemvSide& side, SideBuf& sb) {
    const auto& L = bt_->leaves;
    const std::vector<Block>& oblocks = trans ? cblocks_ : rblocks_;
    const std::vector<int>& ostarts = trans ? cstarts_ : rstarts_;
    std::vector<GemvUnit> units;
    // a longer z task is cut into chunks summed afterwards (spreads long leaves over warps): the
    // 'N' chunk size is the gemv tuner's choice
    const int kMaxUnits = trans ? 16 : tune_zparts_;
    // FP32 'N' y-phase on the tensor-memory kernel when HMAT_B200_TC_Y=1
    const bool tc_y = !trans && std::is_same<T, float>::value && tc_y_enabled();

    // ---- z-phase: 'N' one task per B^T group (z = B^T x_J of its leaves at once, the x rows
    // read once), 'T' one per Rk leaf (z' = A^T x_I over its A panels); long ones cut into
    // chunks; one launch per height class ----
    std::vector<GemvTask> zt[4];
    std::vector<GemvUnit> zunits[4];
    std::vector<GemvZred> zred;
    std::vector<GemvUnit> lu;
    const auto& G = layout_.zgroups;
    const size_t nz = trans ? K.size() : G.size();
    for (size_t t = 0; t < nz; ++t) {
      lu.clear();
      int O, zrow;
      if (!trans) {
        // the group's stacked B^T: h x n column-major
        const ZGroup& g = G[t];
        int xoff = 0;
        const int zc = kTensorN ? mma_unit_cols(g.h, &xoff) : warp_unit_cols_wide(g.h, &xoff);
        px_units(lu, g.base, g.h, g.n, g.col_off, zc, xoff);
        O = g.h;
        zrow = zgroup_row_[0][t];
      } else {
        const GemvRkLeaf& k = K[t];
        const int leaf = rk_leaf[t];
        // z' = A^T x_I: each A panel (len x k) is a transposed piece
        auto br = block_range(rblocks_, rstarts_, k.row_off, k.m);
        for (int b = br.first; b < br.second; ++b)
          ptx_units(lu, layout_.panel[layout_.first[leaf] + (b - br.first)], rblocks_[b].len, k.k, 0,
                    rblocks_[b].off);
        O = k.k;
        zrow = k.zrow_t;
      }
      if (O > 128) throw Error("gemv plan: ranks above 128 are not supported by the streamed kernels");
      // 'N' launches take every height up to 32 in one launch; the tensor-core kernel takes every
      // height up to 64 in one (its tile count is a per-task constant), so one wave covers them
      const int cls = trans ? rank_class(O) : (kTensorN && O <= 64 ? 2 : std::max(1, rank_class(O)));
      // units of one launch must be contiguous in task order: collect them per class
      std::vector<GemvUnit>& cu = zunits[cls];
      if ((int)lu.size() <= kMaxUnits) {
        zt[cls].push_back(GemvTask{O, (int)cu.size(), (int)lu.size(), zrow});
        cu.insert(cu.end(), lu.begin(), lu.end());
      } else {
        const int nparts = ((int)lu.size() + kMaxUnits - 1) / kMaxUnits;
        const int part_row = (int)next_row;
        next_row += (long long)nparts * O;
        for (int pidx = 0; pidx < nparts; ++pidx) {
          const int u0 = pidx * kMaxUnits, u1 = std::min((int)lu.size(), u0 + kMaxUnits);
          GemvTask task{O, (int)cu.size(), u1 - u0, part_row + pidx * O};
          if (zsum_in_kernel(trans)) task.red = (int)zred.size();
          zt[cls].push_back(task);
          cu.insert(cu.end(), lu.begin() + u0, lu.begin() + u1);
        }
        zred.push_back(GemvZred{zrow, O, part_row, nparts});
      }
    }
    for (int c = 0; c < 4; ++c) {
      const int shift = (int)units.size();
      for (auto& t : zt[c]) t.first_unit += shift;
      units.insert(units.end(), zunits[c].begin(), zunits[c].end());
    }
    // ---- y-phase ----
    std::vector<std::vector<int>> per_block(oblocks.size());  // leaves with storage covering each block
    for (int i = 0; i < (int)L.size(); ++i) {
      if (layout_.first[i] < 0) continue;
      auto br = trans ? block_range(oblocks, ostarts, L[i].col_off, L[i].n)
                      : block_range(oblocks, ostarts, L[i].row_off, L[i].m);
      for (int b = br.first; b < br.second; ++b) per_block[b].push_back(i);
    }
    std::vector<int> rk_index(L.size(), -1);
    for (size_t t = 0; t < rk_leaf.size(); ++t) rk_index[rk_leaf[t]] = (int)t;
    std::vector<GemvTask> yt;
    std::vector<int> ybegin;  // 'N': the warps' task ranges, cut here by cost
    int maxlen = 1;
    for (const Block& ob : oblocks) maxlen = std::max(maxlen, ob.len);
    const ClusterTree* otree = trans ? C_ : R_;
    std::vector<int2> yrows(otree->n, int2{0, 0});
    if (!trans) {
      // Each output block's matrix (the y region of the arena) in units of whole columns; the X
      // rows of its columns are the leaves' x rows (full) and z rows (Rk), merged into runs where
      // adjacent, and the zero rows for the padding columns.
      const int RS16 = gemv_rhs_stride((int)sizeof(T), sizeof(T) >= 16 ? 4 : 16);
      const int galign = sizeof(T) >= 16 ? 1 : 16 / (int)sizeof(T);  // columns keeping a piece aligned
      std::vector<int> ublock;  // output block of each y unit
      std::vector<int> colrow;
      const int first_y = (int)units.size();
      for (size_t b = 0; b < oblocks.size(); ++b) {
        const int O = oblocks[b].len, W = layout_.ywidth[b];
        if (W == 0) continue;
        colrow.clear();
        for (int i : per_block[b]) {
          const bool full = L[i].type == 0;
          const int w = full ? L[i].n : ranks[i], row = full ? L[i].col_off : K[rk_index[i]].zrow_n;
          if ((int)colrow.size() != layout_.pcol[layout_.first[i] + (int)b - block_range(rblocks_, rstarts_,
                                                                                          L[i].row_off, L[i].m).first])
            throw Error("gemv plan: block matrix columns out of order");
          for (int j = 0; j < w; ++j) colrow.push_back(row + j);
        }
        const int used = (int)colrow.size();  // at most kYColAlign - 1 = kZeroRows - 1 padding columns
        for (int j = used; j < W; ++j) colrow.push_back(plan_.n_in_max + (j - used));
        int xoff = warp_piece_bytes((int)sizeof(T)), cols;
        if (tc_y)
          cols = kTcCols;
        else if (kTensorN)
          cols = mma_unit_cols(O, &xoff);
        else
          cols = warp_unit_cols_wide(O, &xoff);
        if (tune_yhalf_ && !tc_y) {  // the tuner's narrower units: half the columns, kept aligned
          const int step = kTensorN ? 8 : galign;
          cols = std::max(step, cols / 2 / step * step);
        }
        for (int j0 = 0; j0 < W;) {
          const int want = std::min(cols, W - j0);
          // the columns the unit can take with at most kUnitRuns runs of X rows
          int c = 0, nr = 0;
          while (c < want) {
            if (c == 0 || colrow[j0 + c] != colrow[j0 + c - 1] + 1) {
              if (nr == kUnitRuns) break;
              ++nr;
            }
            ++c;
          }
          if (c < want) c -= c % galign;  // cut short: the next piece must start 16-byte aligned
          if (c <= 0) throw Error("gemv plan: unit without columns");
          GemvUnit u{};
          u.poff = layout_.yblock[b] + (long long)j0 * O;
          u.xrow = colrow[j0];
          u.c = c;
          u.o0 = xoff;
          u.ow = O;
          u.pel = O * c;
          u.shift = (int)(u.poff % kPad);
          if (u.shift) throw Error("gemv plan: misaligned block piece");
          u.nruns = 0;
          for (int j = 0; j < c; ++j) {
            if (j == 0 || colrow[j0 + j] != colrow[j0 + j - 1] + 1) {
              u.run_row[u.nruns] = colrow[j0 + j];
              u.run_len[u.nruns] = 0;
              ++u.nruns;
            }
            ++u.run_len[u.nruns - 1];
          }
          units.push_back(u);
          ublock.push_back((int)b);
          j0 += c;
        }
      }
      // Tasks: the y units cut into one range of about equal cost per warp of the launch, and
      // at block boundaries; a task writes its block's partial rows, summed by the final pass.
      GemvLaunch probe;
      if (tc_y) probe.map = 4;
      else warp_shape(probe, maxlen);
      const int wpc = probe.map == 4 ? 1 : warp_stream_warps_per_cta();
      const int G = launch_ctas(probe.map == 3 ? 8 * probe.rpt : maxlen, false, probe.map != 4, probe.map) * wpc;
      const int nyu = (int)units.size() - first_y;
      std::vector<double> cum(nyu + 1, 0.0);
      for (int v = 0; v < nyu; ++v) {
        const GemvUnit& u = units[first_y + v];
        cum[v + 1] = cum[v] + (double)u.pel + (double)u.c * RS16 + 64;
      }
      const double tot = std::max(cum[nyu], 1.0);
      ybegin.assign(G + 1, 0);
      int w = 0;
      std::vector<int> task_block;
      for (int v = 0; v < nyu;) {
        // the warp of unit v: the last w with cum[v] >= tot * w / G
        while (w + 1 < G && cum[v] >= tot * (w + 1) / G) {
          ++w;
          ybegin[w] = (int)yt.size();
        }
        const double wend = w + 1 < G ? tot * (w + 1) / G : 1e300;
        int v1 = v + 1;
        while (v1 < nyu && ublock[v1] == ublock[v] && cum[v1] < wend) ++v1;
        yt.push_back(GemvTask{oblocks[ublock[v]].len, first_y + v, v1 - v, 0});
        task_block.push_back(ublock[v]);
        v = v1;
      }
      for (++w; w <= G; ++w) ybegin[w] = (int)yt.size();
      // partial-row slots: the tasks of a block (consecutive) take consecutive slots
      std::vector<int> nparts(oblocks.size(), 0), part_row(oblocks.size(), 0);
      for (size_t t = 0; t < yt.size(); ++t) {
        const int b = task_block[t];
        if (nparts[b] == 0) {
          part_row[b] = (int)next_row;
        }
        yt[t].out_row = part_row[b] + nparts[b] * oblocks[b].len;
        nparts[b]++;
        next_row += oblocks[b].len;
      }
      for (size_t b = 0; b < oblocks.size(); ++b) {
        const Block& ob = oblocks[b];
        for (int l = 0; l < ob.len; ++l)
          yrows[otree->perm[ob.off + l]] = int2{part_row[b] + l, (nparts[b] << 8) | ob.len};
      }
    } else {
      // each output block is cut into chunks of at most kYChunkUnits units whose partial rows go
      // to xz; a final pass sums them into y (client order).  The chunks spread the blocks with
      // many leaves over the grid.  The Rk terms come per B^T group: the block's columns of the
      // group's matrix times the group's z' rows.
      const int kYChunkUnits = 16;
      std::vector<std::vector<int>> groups_of(oblocks.size());
      for (size_t gi = 0; gi < G.size(); ++gi) {
        auto br = block_range(oblocks, ostarts, G[gi].col_off, G[gi].n);
        for (int b = br.first; b < br.second; ++b) groups_of[b].push_back((int)gi);
      }
      for (size_t b = 0; b < oblocks.size(); ++b) {
        const Block& ob = oblocks[b];
        const int first = (int)units.size();
        for (int i : per_block[b]) {
          const LeafInfo& l = L[i];
          if (l.type != 0) continue;
          // columns of block b in every row panel of full leaf i
          auto br = block_range(rblocks_, rstarts_, l.row_off, l.m);
          for (int q = br.first; q < br.second; ++q) {
            const int len = rblocks_[q].len;
            ptx_units(units, layout_.panel[layout_.first[i] + (q - br.first)] + (long long)(ob.off - l.col_off) * len,
                      len, ob.len, 0, rblocks_[q].off);
          }
        }
        for (int gi : groups_of[b]) {
          const ZGroup& g = G[gi];
          ptx_units(units, g.base + (long long)(ob.off - g.col_off) * g.h, g.h, ob.len, 0, zgroup_row_[1][gi]);
        }
        const int nu = (int)units.size() - first;
        const int nparts = (nu + kYChunkUnits - 1) / kYChunkUnits;
        const int part_row = (int)next_row;
        next_row += (long long)nparts * ob.len;
        for (int pidx = 0; pidx < nparts; ++pidx) {
          const int u0 = pidx * kYChunkUnits, u1 = std::min(nu, u0 + kYChunkUnits);
          yt.push_back(GemvTask{ob.len, first + u0, u1 - u0, part_row + pidx * ob.len});
        }
        for (int l = 0; l < ob.len; ++l) yrows[otree->perm[ob.off + l]] = int2{part_row + l, (nparts << 8) | ob.len};
      }
    }
    // launches
    side.nz = 0;
    static const int kClassMax[4] = {16, 32, 64, 128};
    for (int c = 0; c < 4; ++c) {
      if (zt[c].empty()) continue;
      int ol, rpt;
      class_shape(c, ol, rpt);
      GemvLaunch& L = side.z[side.nz];
      L = GemvLaunch();
      if (!trans) {
        int om = 1;  // the class's tallest task (FP32 launches hold exactly its tiles)
        for (const GemvTask& t : zt[c]) om = std::max(om, t.O);
        warp_shape(L, kTensorN ? om : kClassMax[c]);
      }
      finish_launch(L, sb, side.nz, zt[c], units, ol, rpt, trans, false);
      side.nz++;
    }
    const int rpt = maxlen <= 32 ? 1 : (maxlen <= 64 ? 2 : 4);
    side.y = GemvLaunch();
    if (tc_y)
      side.y.map = 4;
    else if (!trans)
      warp_shape(side.y, maxlen);
    finish_launch(side.y, sb, GemvSide::kMaxLaunch, yt, units, 32, rpt, trans, false, trans ? nullptr : &ybegin);
    sb.units.upload(units, stream_);
    side.units = sb.units.p;
    sb.zred.upload(zred, stream_);
    side.nzred = (int)zred.size();
    side.zred = sb.zred.p;
    side.zfused = zsum_in_kernel(trans);
    sb.zcnt.alloc((size_t)std::max<size_t>(zred.size(), 1));
    HB_CUDA(cudaMemsetAsync(sb.zcnt.p, 0, sb.zcnt.n * sizeof(int), stream_));
    side.zcnt = sb.zcnt.p;
    sb.yrows.upload(yrows, stream_);
    side.nyrows = (int)yrows.size();
    side.yrows = sb.yrows.p;
  }

  void build_plan() {
    const auto& L = bt_->leaves;
    std::vector<GemvFullLeaf> F;
    std::vector<GemvRkLeaf> K;
    std::vector<int> rk_leaf;
    long long goff = 0;
    plan_ = GemvPlan();
    plan_.n_rows = R_->n;
    plan_.n_cols = C_->n;
    plan_.n_in_max = std::max(R_->n, C_->n);
    long long next_row = plan_.n_in_max + kZeroRows;
    for (size_t i = 0; i < L.size(); ++i) {
      if (L[i].type == 0 && layout_.first[i] >= 0) {
        F.push_back(GemvFullLeaf{L[i].row_off, L[i].m, L[i].col_off, L[i].n, goff});
        goff += (long long)L[i].m * L[i].n;
      } else if (L[i].type == 1 && ranks[i] > 0) {
        GemvRkLeaf k{L[i].row_off, L[i].m, L[i].col_off, L[i].n, ranks[i], 0, goff, 0, 0};
        goff += (long long)ranks[i] * (L[i].m + L[i].n);
        K.push_back(k);
        rk_leaf.push_back((int)i);
      }
    }
    // z slots ('N', then 'T') in the order of the B^T groups: a group's z rows are contiguous
    std::vector<int> kidx(L.size(), -1);
    for (size_t t = 0; t < rk_leaf.size(); ++t) kidx[rk_leaf[t]] = (int)t;
    const auto& G = layout_.zgroups;
    zgroup_row_[0].assign(G.size(), 0);
    zgroup_row_[1].assign(G.size(), 0);
    for (int side = 0; side < 2; ++side)
      for (size_t gi = 0; gi < G.size(); ++gi) {
        zgroup_row_[side][gi] = (int)next_row;
        for (int i : G[gi].leaves) {
          GemvRkLeaf& k = K[kidx[i]];
          (side == 0 ? k.zrow_n : k.zrow_t) = (int)next_row;
          next_row += k.k;
        }
      }
    if (!d_perm_rows_.p || !d_perm_cols_.p) throw Error("gemv plan: cluster permutations are not on the device");
    plan_.perm_rows = d_perm_rows_.p;
    plan_.perm_cols = d_perm_cols_.p;
    std::vector<int> inv(R_->n);
    for (int i = 0; i < R_->n; ++i) inv[R_->perm[i]] = i;
    d_iperm_rows_.upload(inv, stream_);
    inv.assign(C_->n, 0);
    for (int i = 0; i < C_->n; ++i) inv[C_->perm[i]] = i;
    d_iperm_cols_.upload(inv, stream_);
    HB_CUDA(cudaStreamSynchronize(stream_));
    plan_.iperm_rows = d_iperm_rows_.p;
    plan_.iperm_cols = d_iperm_cols_.p;
    plan_.arena = arena_.p;
    g_full_.upload(F, stream_);
    g_rk_.upload(K, stream_);
    plan_.full = g_full_.p;
    plan_.rk = g_rk_.p;
    plan_.nfull = (int)F.size();
    plan_.nrk = (int)K.size();
    build_side(false, K, rk_leaf, next_row, plan_.side[0], side_buf_[0]);
    build_side(true, K, rk_leaf, next_row, plan_.side[1], side_buf_[1]);
    plan_.xz_rows = next_row;
    if (next_row >= (1LL << 31)) throw Error("gemv plan: z buffer too large");
  }

  // Gemv tuner.  Two knobs of the 'N' schedule: the size of the chunks long z tasks are cut into
  // (8, 16 or 32 units: finer chunks spread long groups over more warps, coarser ones write
  // fewer partial rows) and the width of the y-phase units (the widest that fit a stage, or
  // half of it: more, shorter units).  For matrices whose leaves take at least 64 MB, each
  // candidate schedule is built and its z- and y-phases timed on one product (CUDA events, the
  // second of two runs); the fastest chunk size, then the fastest width, are kept and cached for
  // the process by (scalar type, height class of the output blocks).  HMAT_B200_GEMV_TUNE=0
  // keeps the defaults (16, widest); =2 samples any matrix and bypasses the cache (tests).
  int tune_zparts_ = 16;
  bool tune_yhalf_ = false;

  static int gemv_tuning_mode() {
    const char* s = getenv("HMAT_B200_GEMV_TUNE");
    if (!s || !*s) return 1;
    return s[0] == '0' ? 0 : (s[0] == '2' ? 2 : 1);
  }

  // Device ms of the z- and y-phases of one 'N' product with the current schedule.
  void time_phases(double* zms, double* yms) {
    const int nr = std::max(1, std::min(16, kTensorN ? 16 : (sizeof(T) >= 16 ? 4 : 16)));
    DevArray<T> xb, yb;
    xb.alloc((size_t)C_->n * nr);
    yb.alloc((size_t)R_->n * nr);
    HB_CUDA(cudaMemsetAsync(xb.p, 0, xb.n * sizeof(T), stream_));
    xz_.ensure(xz_elems());
    GemvTiming tm;
    for (int i = 0; i < 4; ++i) HB_CUDA(cudaEventCreate(&tm.ev[i]));
    for (int rep = 0; rep < 2; ++rep)
      launch_gemv<T>(plan_, 'N', nr, one<T>(), zero<T>(), xb.p, yb.p, xz_.p, err_.p, stream_, &tm);
    cudaError_t le = cudaGetLastError(), se = cudaStreamSynchronize(stream_);
    float a = 0, b = 0;
    if (le == cudaSuccess && se == cudaSuccess) {
      cudaEventElapsedTime(&a, tm.ev[1], tm.ev[2]);
      cudaEventElapsedTime(&b, tm.ev[2], tm.ev[3]);
    }
    for (int i = 0; i < 4; ++i) cudaEventDestroy(tm.ev[i]);
    HB_CUDA(le);
    HB_CUDA(se);
    check_err_flag();
    *zms = a;
    *yms = b;
  }

  void tune_gemv_plan() {
    gemv_tuned = 0;
    gemv_choice[0] = tune_zparts_ = 16;
    gemv_choice[1] = 0;
    tune_yhalf_ = false;
    for (double& v : gemv_rate) v = 0.0;
    const int mode = gemv_tuning_mode();
    if (mode == 0) return;
    const long long bytes = layout_.total * (long long)sizeof(T);
    if (mode == 1 && bytes < (64LL << 20)) return;
    int maxlen = 1;
    for (const Block& b : rblocks_) maxlen = std::max(maxlen, b.len);
    const auto key = std::make_tuple((int)sizeof(T) * 2 + (Traits<T>::is_complex ? 1 : 0), (maxlen + 15) / 16, 0, 0);
    if (mode == 1) {
      std::lock_guard<std::mutex> g(g_tune_mu);
      auto it = g_gemv_tune_cache.find(key);
      if (it != g_gemv_tune_cache.end()) {
        tune_zparts_ = it->second.first;
        tune_yhalf_ = it->second.second;
        gemv_choice[0] = tune_zparts_;
        gemv_choice[1] = tune_yhalf_ ? 1 : 0;
        gemv_tuned = 2;
        build_plan();
        return;
      }
    }
    static const int kZparts[3] = {8, 16, 32};
    double best_z = 1e300;
    int zp = 16;
    for (int i = 0; i < 3; ++i) {
      tune_zparts_ = kZparts[i];
      tune_yhalf_ = false;
      build_plan();
      double z, y;
      time_phases(&z, &y);
      gemv_rate[i] = z;
      if (i == 0 || z < best_z) {
        best_z = z;
        zp = kZparts[i];
      }
      if (kZparts[i] == 16) gemv_rate[3] = y;  // the widest units' y-phase
    }
    tune_zparts_ = zp;
    tune_yhalf_ = true;
    build_plan();
    double z, yh;
    time_phases(&z, &yh);
    gemv_rate[4] = yh;
    tune_yhalf_ = yh < gemv_rate[3];
    if (!tune_yhalf_) build_plan();
    gemv_choice[0] = tune_zparts_;
    gemv_choice[1] = tune_yhalf_ ? 1 : 0;
    gemv_tuned = 1;
    if (mode == 1) {
      std::lock_guard<std::mutex> g(g_tune_mu);
      g_gemv_tune_cache[key] = std::make_pair(tune_zparts_, tune_yhalf_);
    }
  }

  const ClusterTree* R_;
  const ClusterTree* C_;
  const BlockTree* bt_;
  std::vector<Block> rblocks_, cblocks_;
  std::vector<int> rstarts_, cstarts_;
  cudaStream_t stream_ = nullptr;
  cudaStream_t stream2_ = nullptr;  // runs the tall-skinny truncation beside the CTA kernel
  cudaStream_t stream3_ = nullptr;  // runs the 512-thread ACA beside the other ACA kernels
  cudaStream_t stream4_ = nullptr;  // runs the 64-thread ACA beside the other ACA kernels
  cudaStream_t stream5_ = nullptr;  // runs the 256-thread ACA beside the other ACA kernels
  cudaEvent_t ev_[8];
  cudaEvent_t fork_[2 * kAcaShapes];
  cudaEvent_t tune_ev_[2 * kTuneRuns];  // brackets of the autotuner's sample runs
  KernelParams kp_{};
  std::vector<double> strata_;  // a multi-strata kernel: a_0 .. a_{S-1}, w_0 .. w_{S-1}
  DevArray<double> d_strata_;
  int svd_below_ = 0;
  Points pts_{};
  DevArray<double> d_pts_;
  DevArray<double> d_prm_;  // per-point kernel parameter (cluster order), when the points carry one
  DevArray<int> d_perm_rows_, d_perm_cols_;
  DevArray<int> d_iperm_rows_, d_iperm_cols_;  // client -> cluster order (the gemv's gather)
  std::vector<long long> piece_loff_;  // per Rk leaf: offset of its factors in its piece (assembly)
  std::vector<int> piece_of_;
  std::vector<Piece> pieces_;
  DevArray<T> arena_;
  Layout layout_;
  DevArray<GemvFullLeaf> g_full_;
  DevArray<GemvRkLeaf> g_rk_;
  SideBuf side_buf_[2];
  std::vector<int> zgroup_row_[2];  // first z row of each B^T group, 'N' and 'T' 
  GemvPlan plan_;
  DevArray<T> xz_, rz_, stage_x_, stage_y_;
  DevArray<GemvStatus> err_;       // status block of this matrix's products (flag, wait bound)
  GemvStatus* h_err_ = nullptr;    // pinned host copy
  cudaGraphExec_t gexec_ = nullptr;
  GraphKey gkey_;
};

}  // namespace

std::unique_ptr<EngineBase> make_engine(int value_type, const ClusterTree* rows, const ClusterTree* cols,
                                        const BlockTree* bt) {
  switch (value_type) {
    case 0: return std::unique_ptr<EngineBase>(new Engine<float>(rows, cols, bt));
    case 1: return std::unique_ptr<EngineBase>(new Engine<double>(rows, cols, bt));
    case 2: return std::unique_ptr<EngineBase>(new Engine<cfloat>(rows, cols, bt));
    case 3: return std::unique_ptr<EngineBase>(new Engine<cdouble>(rows, cols, bt));
    default: throw Error("unknown value type");
  }
}

}  // namespace hmatb200
