// B200 engine: device residency and phase orchestration (see engine.h).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>

#include "engine.h"
#include "gemv_plan.h"
#include "kernels.h"

#define HB_CUDA(x)                                                                                  \
  do {                                                                                              \
    cudaError_t e_ = (x);                                                                           \
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
};

inline long long pad32(long long x) { return (x + 31) & ~31LL; }

// Workspace budget of the ACA phase (bytes); batches of admissible leaves are sized to it.
size_t workspace_budget() {
  const char* s = getenv("HMAT_B200_WORKSPACE_MB");
  long long mb = s ? atoll(s) : 8192;
  if (mb < 64) mb = 64;
  return (size_t)mb << 20;
}
// Initial ACA rank capacity per leaf; leaves that reach it are rerun with twice as much.
int initial_kcap() {
  const char* s = getenv("HMAT_B200_ACA_KCAP");
  int k = s ? atoi(s) : 48;
  return k < 4 ? 4 : k;
}

template <typename T>
class Engine : public EngineBase {
  struct SideBufs;
  struct Piece;

 public:
  Engine(const ClusterTree* rows, const ClusterTree* cols, const BlockTree* bt) : R_(rows), C_(cols), bt_(bt) {
    HB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    for (auto& e : ev_) HB_CUDA(cudaEventCreate(&e));
    ranks.assign(bt_->leaves.size(), -1);
    for (size_t i = 0; i < bt_->leaves.size(); ++i)
      if (bt_->leaves[i].type == 1) ranks[i] = 0;
  }
  ~Engine() override {
    if (gexec_) cudaGraphExecDestroy(gexec_);
    for (auto& e : ev_) cudaEventDestroy(e);
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
    upload_points(a);
    const auto& L = bt_->leaves;
    const int nleaves = (int)L.size();
    full_off_.assign(nleaves, -1);
    rk_off_.assign(nleaves, -1);

    // ---- full leaves ----
    std::vector<FullLeafDesc> fd;
    long long fel = 0;
    for (int i = 0; i < nleaves; ++i) {
      if (L[i].type != 0 || L[i].m == 0 || L[i].n == 0) continue;
      FullLeafDesc d{L[i].row_off, L[i].m, L[i].col_off, L[i].n, fel};
      full_off_[i] = fel;
      fel += pad32((long long)L[i].m * L[i].n);
      fd.push_back(d);
    }
    full_arena_.alloc((size_t)std::max(fel, 1LL));
    full_elems_ = fel;
    DevArray<FullLeafDesc> d_fd;
    d_fd.upload(fd, stream_);
    HB_CUDA(cudaEventRecord(ev_[0], stream_));
    launch_assemble_full<T>(d_fd.p, (int)fd.size(), kp_, pts_, full_arena_.p, stream_);
    HB_CUDA(cudaGetLastError());
    HB_CUDA(cudaEventRecord(ev_[1], stream_));
    HB_CUDA(cudaStreamSynchronize(stream_));
    float ms = 0;
    HB_CUDA(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
    times_ms[0] = ms;

    // ---- admissible leaves ----
    assemble_rk(method, eps_aca, eps_trunc, svd_below);
    build_plan();
    HB_CUDA(cudaStreamSynchronize(stream_));
    assembled = true;
  }

  // ------------------------------------------------------------------------------
  void gemv_device(char trans, const void* alpha, const void* x, const void* beta, void* y, int nrhs,
                   cudaStream_t user_stream) override {
    check_gemv_args(trans, nrhs);
    if (nrhs == 0) return;
    const T a = *(const T*)alpha, b = *(const T*)beta;
    x_rm_.ensure((size_t)std::max(R_->n, C_->n) * 16);
    zbuf_.ensure((size_t)std::max(plan_.z_elems, 16LL));
    GraphKey key{trans, nrhs, x, y};
    memcpy(key.ab, &a, sizeof(T));
    memcpy(key.ab + sizeof(T), &b, sizeof(T));
    if (!gexec_ || memcmp(&key, &gkey_, sizeof(GraphKey)) != 0) {
      if (gexec_) {
        cudaGraphExecDestroy(gexec_);
        gexec_ = nullptr;
      }
      cudaGraph_t g;
      HB_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      launch_gemv<T>(plan_, trans, nrhs, a, b, (const T*)x, (T*)y, x_rm_.p, zbuf_.p, zbuf_.p, stream_);
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
    gemv_timed_ = true;
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
    HB_CUDA(cudaStreamSynchronize(stream_));
    HB_CUDA(cudaGetLastError());
    float ms = 0;
    if (cudaEventElapsedTime(&ms, ev_[6], ev_[7]) == cudaSuccess) times_ms[3] = ms;
  }

  // ------------------------------------------------------------------------------
  long long leaf_payload(int leaf, void* out) override {
    if (!assembled || leaf < 0 || leaf >= (int)bt_->leaves.size()) return -1;
    const LeafInfo& L = bt_->leaves[leaf];
    long long cnt = 0;
    const T* src = nullptr;
    if (L.type == 0) {
      if (full_off_[leaf] < 0) return 0;
      cnt = (long long)L.m * L.n;
      src = full_arena_.p + full_off_[leaf];
    } else {
      if (ranks[leaf] <= 0) return 0;
      cnt = (long long)ranks[leaf] * (L.m + L.n);
      src = rk_arena_.p + rk_off_[leaf];
    }
    HB_CUDA(cudaMemcpy(out, src, cnt * sizeof(T), cudaMemcpyDeviceToHost));
    return cnt;
  }

  void arenas(void** full, long long* full_elems, void** rk, long long* rk_elems, long long* offsets) override {
    if (full) *full = full_arena_.p;
    if (full_elems) *full_elems = full_elems_;
    if (rk) *rk = rk_arena_.p;
    if (rk_elems) *rk_elems = rk_elems_;
    if (offsets)
      for (size_t i = 0; i < bt_->leaves.size(); ++i)
        offsets[i] = bt_->leaves[i].type == 0 ? full_off_[i] : rk_off_[i];
  }

  void leaf_gradients(const void* x, const void* r, int nrhs, void* gfull, void* grk, bool accumulate,
                      cudaStream_t user_stream) override {
    if (!assembled) throw Error("matrix is not assembled");
    if (Traits<T>::is_complex) throw Error("leaf gradients are implemented for real value types");
    if (nrhs < 1 || nrhs > 16) throw Error("leaf gradients take 1 to 16 right-hand sides");
    const size_t nmax = (size_t)std::max(R_->n, C_->n);
    x_rm_.ensure(nmax * 16);
    r_rm_.ensure(nmax * 16);
    zbuf_.ensure((size_t)std::max(plan_.z_elems, 16LL));
    zbuf2_.ensure((size_t)std::max(plan_.z_elems, 16LL));
    cudaStream_t s = user_stream ? user_stream : stream_;
    launch_leaf_gradients<T>(plan_, nrhs, (const T*)x, (const T*)r, x_rm_.p, r_rm_.p, zbuf_.p, zbuf2_.p, (T*)gfull,
                             (T*)grk, accumulate, s);
    HB_CUDA(cudaGetLastError());
  }

  void profile_gemv(char trans, const void* x, void* y, int nrhs, double* ms3, double* bytes3) override {
    check_gemv_args(trans, nrhs);
    if (nrhs < 1 || nrhs > 16) throw Error("profile_gemv takes 1 to 16 right-hand sides");
    x_rm_.ensure((size_t)std::max(R_->n, C_->n) * 16);
    zbuf_.ensure((size_t)std::max(plan_.z_elems, 16LL));
    GemvTiming tm;
    for (int i = 0; i < 4; ++i) HB_CUDA(cudaEventCreate(&tm.ev[i]));
    const T one_v = one<T>(), zero_v = zero<T>();
    launch_gemv<T>(plan_, trans, nrhs, one_v, zero_v, (const T*)x, (T*)y, x_rm_.p, zbuf_.p, zbuf_.p, stream_, &tm);
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
    ms3[0] = a;
    ms3[1] = b;
    ms3[2] = c;
    // algorithmic bytes: x read + x_rm write; B (A for 'T') factors; full leaves, A (B)
    // factors and the y write
    const double s = sizeof(T);
    const auto& L = bt_->leaves;
    double full = 0, fa = 0, fb = 0;
    for (size_t i = 0; i < L.size(); ++i) {
      if (L[i].type == 0 && full_off_[i] >= 0) full += (double)L[i].m * L[i].n;
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

  size_t gemv_scratch_bytes() const override {
    const size_t xr = (size_t)std::max(R_->n, C_->n) * 16 * sizeof(T);
    const size_t z = (size_t)std::max(plan_.z_elems, 16LL) * sizeof(T);
    return ((xr + 255) & ~(size_t)255) + z;
  }

  void gemv_device_with_scratch(char trans, const void* alpha, const void* x, const void* beta, void* y, int nrhs,
                                cudaStream_t stream, void* scratch, size_t scratch_bytes) override {
    check_gemv_args(trans, nrhs);
    if (nrhs == 0) return;
    if (gemv_scratch_bytes() > scratch_bytes) throw Error("scratch buffer too small for this matrix");
    const size_t xr = (size_t)std::max(R_->n, C_->n) * 16 * sizeof(T);
    T* x_rm = (T*)scratch;
    T* z = (T*)((char*)scratch + ((xr + 255) & ~(size_t)255));
    launch_gemv<T>(plan_, trans, nrhs, *(const T*)alpha, *(const T*)beta, (const T*)x, (T*)y, x_rm, z, z,
                   stream ? stream : stream_);
    HB_CUDA(cudaGetLastError());
  }

  void retruncate(double eps) override {
    (void)eps;
    throw Error("re-truncation of an assembled matrix is not available yet");
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

  void check_gemv_args(char trans, int nrhs) {
    if (!assembled) throw Error("matrix is not assembled");
    if (trans != 'N' && trans != 'T' && trans != 'C') throw Error("gemv: trans must be 'N', 'T' or 'C'");
    if (nrhs < 0) throw Error("gemv: negative number of right-hand sides");
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
  }

  struct RkJob {
    int leaf;
    int kcap;
    bool svd;
  };

  // Runs ACA (or the dense-SVD fill) and the truncation on one batch of admissible
  // leaves; leaves that ran out of rank capacity are returned in `retry`, the others are
  // compacted into a new piece.
  void run_batch(const std::vector<RkJob>& jobs, double eps_aca, double eps_trunc, std::vector<RkJob>& retry) {
    const auto& L = bt_->leaves;
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
    // cost-sorted orders (largest first) for the ACA and dense-fill groups
    std::vector<int> aca_order, svd_order;
    for (int b = 0; b < nb; ++b) (jobs[b].svd ? svd_order : aca_order).push_back(b);
    auto cost = [&](int b) { return (double)(desc[b].m + desc[b].n) * std::min(desc[b].m, desc[b].n); };
    std::stable_sort(aca_order.begin(), aca_order.end(), [&](int x, int y) { return cost(x) > cost(y); });
    DevArray<RkLeafDesc> d_desc;
    d_desc.upload(desc, stream_);
    DevArray<T> d_ws;
    d_ws.alloc((size_t)ws);
    DevArray<unsigned char> d_flags;
    d_flags.alloc((size_t)std::max(fl, 1LL));
    DevArray<int> d_ranks, d_status, d_counter, d_aca_order, d_svd_order;
    d_ranks.alloc(nb);
    d_status.alloc(nb);
    d_counter.alloc(1);
    HB_CUDA(cudaMemsetAsync(d_ranks.p, 0, nb * sizeof(int), stream_));
    HB_CUDA(cudaMemsetAsync(d_status.p, 0, nb * sizeof(int), stream_));
    d_aca_order.upload(aca_order, stream_);
    d_svd_order.upload(svd_order, stream_);

    HB_CUDA(cudaEventRecord(ev_[2], stream_));
    if (!aca_order.empty()) {
      HB_CUDA(cudaMemsetAsync(d_counter.p, 0, sizeof(int), stream_));
      launch_aca<T>(d_desc.p, d_aca_order.p, (int)aca_order.size(), kp_, pts_, eps_aca, d_ws.p, d_flags.p,
                    d_ranks.p, d_status.p, d_counter.p, max_cap, persistent_grid(8), stream_);
      HB_CUDA(cudaGetLastError());
    }
    if (!svd_order.empty()) {
      launch_dense_to_rk<T>(d_desc.p, d_svd_order.p, (int)svd_order.size(), kp_, pts_, d_ws.p, d_ranks.p,
                            d_status.p, stream_);
      HB_CUDA(cudaGetLastError());
    }
    HB_CUDA(cudaEventRecord(ev_[3], stream_));
    std::vector<int> h_status(nb), h_ranks(nb);
    HB_CUDA(cudaMemcpyAsync(h_status.data(), d_status.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    HB_CUDA(cudaMemcpyAsync(h_ranks.data(), d_ranks.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    HB_CUDA(cudaStreamSynchronize(stream_));
    float ms = 0;
    HB_CUDA(cudaEventElapsedTime(&ms, ev_[2], ev_[3]));
    times_ms[1] += ms;

    std::vector<int> good;
    int max_k = 1;
    for (int b = 0; b < nb; ++b) {
      if (h_status[b] == kLeafAcaCapacity) {
        const LeafInfo& l = L[jobs[b].leaf];
        RkJob j = jobs[b];
        j.kcap = std::min(std::min(l.m, l.n), 2 * j.kcap);
        retry.push_back(j);
        h_ranks[b] = 0;
        continue;
      }
      if (h_status[b] != kLeafOk) throw Error("device compression failed on a leaf (status " +
                                              std::to_string(h_status[b]) + ")");
      if (h_ranks[b] > 0) good.push_back(b);
      max_k = std::max(max_k, h_ranks[b]);
    }
    auto tcost = [&](int b) { return (double)(desc[b].m + desc[b].n) * h_ranks[b] * h_ranks[b]; };
    std::stable_sort(good.begin(), good.end(), [&](int x, int y) { return tcost(x) > tcost(y); });

    HB_CUDA(cudaEventRecord(ev_[4], stream_));
    if (!good.empty()) {
      typedef typename Traits<T>::wide W;
      const long long slab = truncate_slab_elems<T>(max_m, max_n, max_k);
      const size_t budget = workspace_budget();
      long long grid = std::min<long long>((long long)good.size(), persistent_grid(2));
      grid = std::max(1LL, std::min<long long>(grid, (long long)(budget / (slab * sizeof(W)))));
      DevArray<W> d_scratch;
      d_scratch.alloc((size_t)(grid * slab));
      DevArray<int> d_good;
      if (!svd_order.empty()) {
        // SVD of the dense blocks at the compression epsilon, then the regular truncation
        std::vector<int> svd_good;
        for (int b : good)
          if (jobs[b].svd) svd_good.push_back(b);
        if (!svd_good.empty()) {
          d_good.upload(svd_good, stream_);
          HB_CUDA(cudaMemsetAsync(d_counter.p, 0, sizeof(int), stream_));
          launch_truncate<T>(d_desc.p, d_good.p, (int)svd_good.size(), eps_aca, d_ws.p, d_ranks.p, d_status.p,
                             d_counter.p, d_scratch.p, slab, (int)grid, stream_);
          HB_CUDA(cudaGetLastError());
        }
      }
      d_good.upload(good, stream_);
      HB_CUDA(cudaMemsetAsync(d_counter.p, 0, sizeof(int), stream_));
      launch_truncate<T>(d_desc.p, d_good.p, (int)good.size(), eps_trunc, d_ws.p, d_ranks.p, d_status.p,
                         d_counter.p, d_scratch.p, slab, (int)grid, stream_);
      HB_CUDA(cudaGetLastError());
    }
    // overflowed leaves must not be compacted
    HB_CUDA(cudaMemcpyAsync(h_ranks.data(), d_ranks.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    HB_CUDA(cudaMemcpyAsync(h_status.data(), d_status.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream_));
    HB_CUDA(cudaStreamSynchronize(stream_));
    for (int b = 0; b < nb; ++b)
      if (h_status[b] == kLeafAcaCapacity) h_ranks[b] = 0;
    HB_CUDA(cudaMemcpyAsync(d_ranks.p, h_ranks.data(), nb * sizeof(int), cudaMemcpyHostToDevice, stream_));
    std::vector<long long> dst(nb, 0);
    long long pe = 0;
    for (int b = 0; b < nb; ++b) {
      dst[b] = pe;
      if (h_ranks[b] > 0) pe += pad32((long long)h_ranks[b] * (desc[b].m + desc[b].n));
    }
    Piece piece;
    piece.arena.alloc((size_t)std::max(pe, 1LL));
    piece.elems = pe;
    DevArray<long long> d_dst;
    d_dst.upload(dst, stream_);
    launch_compact<T>(d_desc.p, nb, d_ws.p, d_ranks.p, d_dst.p, piece.arena.p, stream_);
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
      rk_off_[leaf] = h_ranks[b] > 0 ? dst[b] : -1;
      if (h_status[b] == kLeafSvdNoConverge) svd_warnings_++;
    }
    pieces_.push_back(std::move(piece));
  }

  void assemble_rk(int method, double eps_aca, double eps_trunc, int svd_below) {
    (void)method;
    const auto& L = bt_->leaves;
    const int nleaves = (int)L.size();
    times_ms[1] = times_ms[2] = 0;
    piece_of_.assign(nleaves, -1);
    pieces_.clear();
    svd_warnings_ = 0;
    std::vector<RkJob> queue;
    const int k0 = initial_kcap();
    for (int i = 0; i < nleaves; ++i) {
      if (L[i].type != 1) continue;
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
        run_batch(batch, eps_aca, eps_trunc, retry);
      }
      queue.swap(retry);
    }
    // concatenate the pieces into one arena
    std::vector<long long> base(pieces_.size(), 0);
    long long tot = 0;
    for (size_t p = 0; p < pieces_.size(); ++p) {
      base[p] = tot;
      tot += pad32(pieces_[p].elems);
    }
    rk_arena_.alloc((size_t)std::max(tot, 1LL));
    rk_elems_ = tot;
    for (size_t p = 0; p < pieces_.size(); ++p)
      if (pieces_[p].elems)
        HB_CUDA(cudaMemcpyAsync(rk_arena_.p + base[p], pieces_[p].arena.p, pieces_[p].elems * sizeof(T),
                                cudaMemcpyDeviceToDevice, stream_));
    for (int i = 0; i < nleaves; ++i)
      if (L[i].type == 1 && piece_of_[i] >= 0) rk_off_[i] += base[piece_of_[i]];
    HB_CUDA(cudaStreamSynchronize(stream_));
    pieces_.clear();
  }

  // ------------------------------------------------------------------------------
  void build_side(bool trans, const std::vector<GemvFullLeaf>& F, const std::vector<GemvRkLeaf>& K,
                  long long zbase, SideBufs& sb, GemvSide& side) {
    const ClusterTree& out = trans ? *C_ : *R_;
    const int nb = (int)out.leaf_nodes.size();
    std::vector<int> start(nb);
    for (int b = 0; b < nb; ++b) start[b] = out.nodes[out.leaf_nodes[b]].offset;
    std::vector<std::vector<GemvYEntry>> lists(nb);
    auto add_range = [&](int type, int idx, int off, int len) {
      int b = (int)(std::upper_bound(start.begin(), start.end(), off) - start.begin()) - 1;
      for (; b < nb && start[b] < off + len; ++b) {
        GemvYEntry e{type, idx, start[b] - off, 0};
        lists[b].push_back(e);
      }
    };
    for (int f = 0; f < (int)F.size(); ++f)
      add_range(0, f, trans ? F[f].col_off : F[f].row_off, trans ? F[f].n : F[f].m);
    for (int k = 0; k < (int)K.size(); ++k)
      add_range(1, k, trans ? K[k].col_off : K[k].row_off, trans ? K[k].n : K[k].m);
    std::vector<GemvYBlock> blocks;
    std::vector<GemvYEntry> entries;
    int maxlen = 1;
    for (int b = 0; b < nb; ++b) {
      const ClusterNode& nd = out.nodes[out.leaf_nodes[b]];
      GemvYBlock blk{nd.offset, nd.size, (int)entries.size(), (int)lists[b].size()};
      entries.insert(entries.end(), lists[b].begin(), lists[b].end());
      blocks.push_back(blk);
      maxlen = std::max(maxlen, nd.size);
    }
    // z items: long leaves are cut into chunks whose partials are summed afterwards
    const int kChunk = 512;
    std::vector<GemvZItem> items;
    std::vector<int> multi, mfirst, mcount;
    long long zpos = zbase;
    for (int k = 0; k < (int)K.size(); ++k) {
      const int len = trans ? K[k].m : K[k].n;
      if (len <= kChunk) {
        items.push_back(GemvZItem{k, 0, len, 0, K[k].zoff});
      } else {
        multi.push_back(k);
        mfirst.push_back((int)items.size());
        int cnt = 0;
        for (int s = 0; s < len; s += kChunk, ++cnt) {
          items.push_back(GemvZItem{k, s, std::min(kChunk, len - s), 0, zpos});
          zpos += (long long)K[k].k * 16;
        }
        mcount.push_back(cnt);
      }
    }
    plan_.z_elems = std::max(plan_.z_elems, zpos);
    sb.blocks.upload(blocks, stream_);
    sb.entries.upload(entries, stream_);
    sb.items.upload(items, stream_);
    sb.multi.upload(multi, stream_);
    sb.mfirst.upload(mfirst, stream_);
    sb.mcount.upload(mcount, stream_);
    side.nblocks = nb;
    side.blocks = sb.blocks.p;
    side.entries = sb.entries.p;
    side.nzitems = (int)items.size();
    side.zitems = sb.items.p;
    side.nmulti = (int)multi.size();
    side.multi = sb.multi.p;
    side.mfirst = sb.mfirst.p;
    side.mcount = sb.mcount.p;
    int gs = ((maxlen + 31) / 32) * 32;
    side.GS = std::min(gs, 128);
  }

  void build_plan() {
    const auto& L = bt_->leaves;
    std::vector<GemvFullLeaf> F;
    std::vector<GemvRkLeaf> K;
    long long zoff = 0;
    for (size_t i = 0; i < L.size(); ++i) {
      if (L[i].type == 0 && full_off_[i] >= 0) {
        F.push_back(GemvFullLeaf{L[i].row_off, L[i].m, L[i].col_off, L[i].n, full_off_[i]});
      } else if (L[i].type == 1 && ranks[i] > 0) {
        GemvRkLeaf k{L[i].row_off, L[i].m, L[i].col_off, L[i].n, ranks[i], 0, rk_off_[i], zoff};
        zoff += (long long)ranks[i] * 16;
        K.push_back(k);
      }
    }
    plan_ = GemvPlan();
    plan_.n_rows = R_->n;
    plan_.n_cols = C_->n;
    plan_.perm_rows = d_perm_rows_.p;
    plan_.perm_cols = d_perm_cols_.p;
    g_full_.upload(F, stream_);
    g_rk_.upload(K, stream_);
    plan_.full = g_full_.p;
    plan_.rk = g_rk_.p;
    plan_.nfull = (int)F.size();
    plan_.nrk = (int)K.size();
    plan_.full_arena = full_arena_.p;
    plan_.rk_arena = rk_arena_.p;
    plan_.z_elems = zoff;
    build_side(false, F, K, zoff, side_n_, plan_.side_n);
    build_side(true, F, K, zoff, side_t_, plan_.side_t);
  }

  struct Piece {
    DevArray<T> arena;
    long long elems = 0;
  };
  struct SideBufs {
    DevArray<GemvYBlock> blocks;
    DevArray<GemvYEntry> entries;
    DevArray<GemvZItem> items;
    DevArray<int> multi, mfirst, mcount;
  };

  const ClusterTree* R_;
  const ClusterTree* C_;
  const BlockTree* bt_;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev_[8];
  KernelParams kp_{};
  Points pts_{};
  DevArray<double> d_pts_;
  DevArray<int> d_perm_rows_, d_perm_cols_;
  std::vector<long long> full_off_, rk_off_;
  std::vector<int> piece_of_;
  std::vector<Piece> pieces_;
  DevArray<T> full_arena_, rk_arena_;
  long long full_elems_ = 0, rk_elems_ = 0;
  int svd_warnings_ = 0;
  DevArray<GemvFullLeaf> g_full_;
  DevArray<GemvRkLeaf> g_rk_;
  SideBufs side_n_, side_t_;
  GemvPlan plan_;
  DevArray<T> x_rm_, r_rm_, zbuf_, zbuf2_, stage_x_, stage_y_;
  cudaGraphExec_t gexec_ = nullptr;
  GraphKey gkey_;
  bool gemv_timed_ = false;
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
