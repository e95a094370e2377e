// Device-resident solver: upload of a graph + LDLinv factor, and the solve
// (FP64 PCG, or FP32 PCG inside FP64 iterative refinement) as one CUDA graph
// whose PCG loop is a conditional WHILE node, so a whole solve is one graph
// launch with no host round trip per iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/acgpu.h"
#include "acg_internal.h"
#include "acg_batch.cuh"
#include "acg_dense.cuh"
#include "acg_group.cuh"
#include "acg_serve.cuh"

namespace acg {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct InputError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct DeviceNoMem : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define ACG_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::acg::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " + \
                             __FILE__ + ":" + std::to_string(__LINE__));                    \
  } while (0)

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    free();
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      p = nullptr;
      throw DeviceNoMem("device allocation of " + std::to_string(count * sizeof(T)) + " bytes failed");
    }
    ACG_CUDA(e);
    n = count;
  }
  void upload(const std::vector<T>& h, cudaStream_t s) {
    alloc(h.size());
    if (!h.empty()) ACG_CUDA(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

// One step of a sweep plan: a single wide level (grid launch) or a run of
// thin levels executed by one CTA with the run's values in shared memory.
struct SweepStep {
  int thin;
  int l0, l1;   // levels [l0, l1)
  int v0, v1;   // vertex range of the levels
  int nw;       // forward: leading vertices with in-degree > 32 (a warp each)
  size_t smem;  // thin runs: dynamic shared memory bytes
};

// Graph capture and device (de)allocation are serialised across threads: an
// allocation or free on one thread while another thread captures a stream can
// invalidate that capture.  Graph launches do not take this lock.
std::recursive_mutex g_device_mu;

struct SolverImpl {
  int device = 0;
  cudaStream_t stream = nullptr;
  int n = 0;
  int64_t nnz_l = 0, nnz_f = 0;
  int64_t nnz_fsweep = 0, nnz_bsweep = 0;  // entries the forward / backward sweeps walk
  int nlev = 0;
  int vl_spmv = 8;
  int thin_max_width = 2048;
  size_t smem_optin = 0;
  std::vector<int> lvl_off;        // host copy
  int nseg = 1;                    // graphs in this solver (a group holds several)
  std::vector<int> seg_off;        // graph g = internal vertices [seg_off[g], seg_off[g+1])
  std::vector<int> heavy;          // per level: vertices with forward in-degree > 32
  std::vector<SweepStep> plan[2];  // [0] FP64 values, [1] FP32 values
  int sweep_mode = 0;              // 0 sync-free cooperative sweep, 1 one launch per level
  // narrow tail of the DAG run by one CTA (k_tail): levels [nlev - tail_nl, nlev)
  int tail_nl = 0, tail_v0 = 0, tail_nv = 0;
  int tail_tf0 = 0;                // forward: sync-free tasks [0, tail_tf0), the tail after
  int tail_tb0 = 0;                // backward: the tail first, then sync-free tasks [tail_tb0, ntasks_b)
  DevBuf<int2> tail_lvl_f, tail_lvl_b;
  int ntasks_f = 0, ntasks_b = 0;
  int sweep_blocks[2] = {0, 0};    // co-resident grid of k_sweep per value type
  int poll_mode = 0;
  unsigned spin_limit = kSpinLimit;  // polls before a sweep wait gives up
  double min_inner_tol = 2e-5;       // mixed precision: floor of an inner solve's tolerance
  cudaEvent_t order_ev = nullptr;    // device entry points: after the legacy stream's work
  DevBuf<SweepTask> tasks_f, tasks_b;

  DevBuf<int> perm, lvl_off_d;
  DevBuf<int> iperm;               // external vertex -> internal (the batched gather and scatter)
  DevBuf<int> l_ptr, l_idx, f_ptr, f_idx, b_ptr, b_idx;
  DevBuf<double> l_v64, f_c64, b_c64, g64;
  DevBuf<float> l_v32, f_c32, b_c32, g32;

  // work vectors
  DevBuf<double> b_ext, x_ext, bm, r64, s64, y64, p64, q64, x3_64, xf;
  DevBuf<float> r32, s32, y32, p32, q32, x3_32;
  DevBuf<double> partials;
  PcgState* st = nullptr;    // device
  PcgState* h_st = nullptr;  // pinned host mirror

  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  std::mutex mu;
  unsigned char* noalloc_scratch = nullptr;  // device address of the fixed scratch array

  // groups: several graphs in one solver (nseg > 1), one right-hand side each
  int nchunks = 0;
  DevBuf<SegChunk> chunks;
  DevBuf<int> seg_first, seg_nchunk;
  DevBuf<unsigned int> seg_cnt;
  DevBuf<double> gpartials;
  PcgState* gstates = nullptr;  // per graph (device)
  PcgState* gflags = nullptr;   // group flags (device)
  GroupShared* gsh = nullptr;
  PcgState* h_gstates = nullptr;
  cudaGraphExec_t gexec = nullptr, gexec_mixed = nullptr;

  // batched solves: kp right-hand sides per launch (vertex-major n x kp blocks)
  int batch_kp = 0;  // capacity of the batch buffers
  DevBuf<double> bb_ext[2], bx_ext[2];  // external-order blocks, one pair per slot (slot 1: asynchronous solves)
  DevBuf<double> bbm, br64, bxf, bpartials;
  DevBuf<float> br32, bs32, by32, bp32, bq32, bx3_32;
  DevBuf<double> bs64, by64, bp64, bq64, bx3_64;
  PcgState* bst = nullptr;
  BatchShared* bsh = nullptr;
  PcgState* h_bst = nullptr;
  int bsweep_blocks[2][4] = {};          // [precision][log2(kp/8)]
  int bvec_blocks[2][4] = {};            // [precision][pq, update, yzr, pupdate]: one resident wave
  int bspmv_blocks[2][4] = {};           // batched mat-vec grid: every resident block
  int batch_bps = 0;                     // batched sweep blocks per SM (0 = occupancy limit)
  // dense tail: vertices [dt_v0, n) (levels >= dt_L0) handled by s_T = M w_T,
  // y_T = M^T (g_T s_T) with M = (I - C_TT)^{-1} (K x K, row-major); K = 0: none
  int dt_K = 0, dt_v0 = 0, dt_L0 = 0;
  // values per vertex in the one-vector sweep vectors s and y (FP64, FP32):
  // one 32-byte sector per vertex for the sync-free engine, so values that
  // different SMs write at nearly the same time never share a sector
  int vs64 = 1, vs32 = 1;
  DevBuf<double> dt_M64, dt_part;        // dt_part: partial tiles (chunks x K x columns, as T)
  DevBuf<float> dt_M32;
  size_t dt_part_cols = 0;               // columns dt_part holds
  int ntasks_bb = 0, ntasks_fb = 0;      // task tables of the batched sweeps
  DevBuf<SweepTask> tasks_bb, tasks_fb;
  // per level l: the forward table's tasks of levels <= l, and the backward
  // table's tasks of levels >= l (the backward table walks levels downwards)
  std::vector<int> tfb_upto, tbb_from;
  cudaGraphExec_t bexec[2][2][4] = {};  // [slot][precision][log2(kp/8)]

  // asynchronous batched solves (acg_solve_async): two slots, each with its
  // own external blocks and graphs, so that one request's host copies run
  // while the other request solves.  Copies in run on h2d_stream, copies out
  // on d2h_stream, solves on `stream`.
  struct AsyncSlot {
    cudaEvent_t h2d = nullptr, start = nullptr, done = nullptr, d2h = nullptr;
    PcgState* h_init = nullptr;    // pinned: the request's initial column states
    PcgState* h_out = nullptr;     // pinned: its final column states
    BatchShared* h_bsh = nullptr;  // pinned
    acg_request* owner = nullptr;  // request whose results are not yet collected
  };
  bool async_on = false;
  bool serving = false;  // a serving loop (acg_serve_open) owns the batch buffers
  acg_server* server = nullptr;
  cudaStream_t h2d_stream = nullptr, d2h_stream = nullptr;
  AsyncSlot slots[2];
  int next_slot = 0;

  ~SolverImpl() {
    for (auto& e : exec)
      if (e) cudaGraphExecDestroy(e);
    for (auto& per_slot : bexec)
      for (auto& row : per_slot)
        for (auto& e : row)
          if (e) cudaGraphExecDestroy(e);
    for (AsyncSlot& a : slots) {
      for (cudaEvent_t e : {a.h2d, a.start, a.done, a.d2h})
        if (e) cudaEventDestroy(e);
      if (a.h_init) cudaFreeHost(a.h_init);
      if (a.h_out) cudaFreeHost(a.h_out);
      if (a.h_bsh) cudaFreeHost(a.h_bsh);
    }
    if (h2d_stream) cudaStreamDestroy(h2d_stream);
    if (d2h_stream) cudaStreamDestroy(d2h_stream);
    if (order_ev) cudaEventDestroy(order_ev);
    if (bst) cudaFree(bst);
    if (bsh) cudaFree(bsh);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (gexec_mixed) cudaGraphExecDestroy(gexec_mixed);
    if (gstates) cudaFree(gstates);
    if (gflags) cudaFree(gflags);
    if (gsh) cudaFree(gsh);
    if (h_gstates) cudaFreeHost(h_gstates);
    if (h_bst) cudaFreeHost(h_bst);
    if (st) cudaFree(st);
    if (h_st) cudaFreeHost(h_st);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

int choose_vl(double avg) {
  if (avg <= 2.5) return 2;
  if (avg <= 5.0) return 4;
  if (avg <= 12.0) return 8;
  return 16;
}

// ---- kernel launch helpers (runtime VL -> template) -----------------------

template <typename T>
struct TypedArrays {
  const int *fp, *fi, *bp, *bi, *lp, *li;
  const T *fc, *bc, *g, *lv, *dm;
};

template <typename T>
TypedArrays<T> arrays_of(const SolverImpl& S);
template <>
TypedArrays<double> arrays_of<double>(const SolverImpl& S) {
  return {S.f_ptr.p, S.f_idx.p, S.b_ptr.p, S.b_idx.p, S.l_ptr.p, S.l_idx.p, S.f_c64.p, S.b_c64.p, S.g64.p, S.l_v64.p, S.dt_M64.p};
}
template <>
TypedArrays<float> arrays_of<float>(const SolverImpl& S) {
  return {S.f_ptr.p, S.f_idx.p, S.b_ptr.p, S.b_idx.p, S.l_ptr.p, S.l_idx.p, S.f_c32.p, S.b_c32.p, S.g32.p, S.l_v32.p, S.dt_M32.p};
}

#define ACG_VL_SWITCH(vl, FN, ...)                   \
  switch (vl) {                                      \
    case 2: FN<T, 2>(__VA_ARGS__); break;            \
    case 4: FN<T, 4>(__VA_ARGS__); break;            \
    case 8: FN<T, 8>(__VA_ARGS__); break;            \
    default: FN<T, 16>(__VA_ARGS__); break;          \
  }

template <typename T>
constexpr int plan_index() {
  return sizeof(T) == sizeof(double) ? 0 : 1;
}
template <typename T>
int vstride(const SolverImpl& S) {
  return sizeof(T) == sizeof(double) ? S.vs64 : S.vs32;
}

// Launch with programmatic stream serialisation (PDL): the kernel's prologue
// (constant structure loads) overlaps the previous launch in the stream.
template <typename... KArgs, typename... Args>
void launch_pdl(cudaStream_t s, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ACG_CUDA(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
}

template <typename T, bool kForward>
void enqueue_step(cudaStream_t s, const SolverImpl& S, const SweepStep& st_, const T* aux, const T* sfwd, T* vals,
                  const PcgState* st) {
  const TypedArrays<T> A = arrays_of<T>(S);
  const int* ptr = kForward ? A.fp : A.bp;
  const int* idx = kForward ? A.fi : A.bi;
  const T* coef = kForward ? A.fc : A.bc;
  if (st_.thin) {
    launch_pdl(s, k_thin<T, kForward>, dim3(1), dim3(kThinThreads), st_.smem, st_.l0, st_.l1,
               (const int*)S.lvl_off_d.p, ptr, idx, coef, aux, sfwd, vals, st);
  } else {
    const int nw = kForward ? st_.nw : 0;
    const long long per_warp = 32 / kLightLanes;
    const long long warps = nw + ((long long)(st_.v1 - st_.v0 - nw) + per_warp - 1) / per_warp;
    const int blocks = (int)((warps * 32 + kLevelThreads - 1) / kLevelThreads);
    launch_pdl(s, k_level<T, kForward>, dim3(blocks), dim3(kLevelThreads), 0, st_.v0, st_.v1, nw, ptr, idx, coef,
               aux, sfwd, vals, st);
  }
}

// One sync-free sweep over tasks [t0, t1) as a cooperative launch (all blocks co-resident).
template <typename T, bool kForward>
void enqueue_syncfree(cudaStream_t s, const SolverImpl& S, const T* aux, const T* sfwd, T* out, PcgState* st,
                      int t0, int t1, int vs) {
  if (t1 <= t0) return;
  const TypedArrays<T> A = arrays_of<T>(S);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(S.sweep_blocks[plan_index<T>()]);
  cfg.blockDim = dim3(kSweepThreads);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const SweepTask* tasks = (kForward ? S.tasks_f.p : S.tasks_b.p) + t0;
  ACG_CUDA(cudaLaunchKernelEx(&cfg, k_sweep<T, kForward>, t1 - t0, tasks, kForward ? A.fi : A.bi,
                              kForward ? A.fc : A.bc, aux, sfwd, out, st, S.poll_mode, vs, S.spin_limit));
}

// The narrow tail of the DAG in one CTA.
template <typename T, bool kForward>
void enqueue_tail(cudaStream_t s, const SolverImpl& S, const T* aux, const T* sfwd, T* out, const PcgState* st) {
  const TypedArrays<T> A = arrays_of<T>(S);
  const size_t smem = tail_smem_bytes<T>(S.tail_nv, S.tail_nl);
  k_tail<T, kForward><<<1, kTailThreads, smem, s>>>(
      S.tail_nl, S.tail_v0, S.tail_nv, kForward ? S.tail_lvl_f.p : S.tail_lvl_b.p, kForward ? S.ntasks_f : S.ntasks_b,
      kForward ? S.tasks_f.p : S.tasks_b.p, kForward ? A.fi : A.bi, kForward ? A.fc : A.bc, aux, sfwd, out, st);
}

// The dense tail step of a sweep on kp-column vectors (kp = 1, or 8 * CPL):
// forward s_T = M w_T in place in sv; backward y_T = M^T (g_T s_T).  part
// holds the partial tiles; done (device) ends the step early when set.
template <typename T, int CPL>
void enqueue_dense(cudaStream_t s, const SolverImpl& S, bool fwd, T* sv, T* y, T* part, const int* done,
                   int vs = 1) {
  constexpr int kp = CPL == 0 ? 1 : 8 * CPL;
  const int K = S.dt_K;
  const TypedArrays<T> A = arrays_of<T>(S);
  const int rs = CPL == 0 ? vs : kp;  // row stride of sv and y
  const size_t off = (size_t)S.dt_v0 * rs;
  const dim3 grid(dense_row_tiles(K), dense_chunks(K));
  const T* g = A.g + S.dt_v0;
  if constexpr (CPL == 0) {
    if (fwd) kd1_partial<T, true><<<grid, kDenseThreads, 0, s>>>(K, A.dm, sv + off, g, part, done, vs);
    else kd1_partial<T, false><<<grid, kDenseThreads, 0, s>>>(K, A.dm, sv + off, g, part, done, vs);
  } else {
    if (fwd) kd_partial<T, CPL, true><<<grid, kDenseThreads, 0, s>>>(K, A.dm, sv + off, g, part, done);
    else kd_partial<T, CPL, false><<<grid, kDenseThreads, 0, s>>>(K, A.dm, sv + off, g, part, done);
  }
  ACG_CUDA(cudaGetLastError());
  const int rb = (int)std::min<long long>(kVecBlocks, ((long long)K * kp + kVecThreads - 1) / kVecThreads);
  if (fwd) kd_reduce<T, true><<<rb, kVecThreads, 0, s>>>(K, kp, part, sv + off, done, rs);
  else kd_reduce<T, false><<<rb, kVecThreads, 0, s>>>(K, kp, part, y + off, done, rs);
}

// Forward sweep: s = forward values of r (s must be pending in sync-free mode).
// part: partial tiles of the dense tail (null: the solver's own buffer); vs:
// values per vertex in sv and y (-1: the solver's own layout, vstride<T>).
template <typename T>
void enqueue_forward(cudaStream_t s, const SolverImpl& S, const T* r, T* sv, PcgState* st, T* part = nullptr,
                     bool dense = true, int vs = -1) {
  if (vs < 0) vs = vstride<T>(S);
  if (S.sweep_mode == 0) {
    if (S.tail_nl > 0) {
      enqueue_syncfree<T, true>(s, S, r, (const T*)nullptr, sv, st, 0, S.tail_tf0, vs);
      enqueue_tail<T, true>(s, S, r, (const T*)nullptr, sv, st);
    } else {
      enqueue_syncfree<T, true>(s, S, r, (const T*)nullptr, sv, st, 0, S.ntasks_f, vs);
    }
    if (S.dt_K && dense)
      enqueue_dense<T, 0>(s, S, true, sv, (T*)nullptr, part ? part : reinterpret_cast<T*>(S.dt_part.p), &st->done,
                          vs);
    return;
  }
  for (const SweepStep& step : S.plan[plan_index<T>()]) enqueue_step<T, true>(s, S, step, r, (const T*)nullptr, sv, st);
}
// Backward sweep: y from the forward values s (y pending in sync-free mode).
template <typename T>
void enqueue_backward(cudaStream_t s, const SolverImpl& S, const T* sv, T* y, PcgState* st, T* part = nullptr,
                      bool dense = true, int vs = -1) {
  if (vs < 0) vs = vstride<T>(S);
  const T* g = arrays_of<T>(S).g;
  if (S.sweep_mode == 0) {
    if (S.dt_K && dense)
      enqueue_dense<T, 0>(s, S, false, const_cast<T*>(sv), y, part ? part : reinterpret_cast<T*>(S.dt_part.p),
                          &st->done, vs);
    if (S.tail_nl > 0) {
      enqueue_tail<T, false>(s, S, g, sv, y, st);
      enqueue_syncfree<T, false>(s, S, g, sv, y, st, S.tail_tb0, S.ntasks_b, vs);
    } else {
      enqueue_syncfree<T, false>(s, S, g, sv, y, st, 0, S.ntasks_b, vs);
    }
    return;
  }
  const auto& plan = S.plan[plan_index<T>()];
  for (auto it = plan.rbegin(); it != plan.rend(); ++it) enqueue_step<T, false>(s, S, *it, g, sv, y, st);
}
// y = LDLinv sweeps of r (without the final mean removal); sv is scratch.
template <typename T>
void enqueue_sweeps(cudaStream_t s, const SolverImpl& S, const T* r, T* sv, T* y, PcgState* st, T* part = nullptr,
                    int vs = -1) {
  enqueue_forward<T>(s, S, r, sv, st, part, true, vs);
  enqueue_backward<T>(s, S, sv, y, st, part, true, vs);
}

template <typename T, int VL>
void spmv_pq_vl(cudaStream_t s, const SolverImpl& S, const TypedArrays<T>& A, const T* p, T* q, PcgState* st,
                double eps, LoopCtl ctl) {
  k_spmv_pq<T, VL><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, A.lp, A.li, A.lv, p, q, st, S.partials.p, eps, ctl);
}
template <typename T, int VL>
void true_res_vl(cudaStream_t s, const SolverImpl& S, const double* x, const double* bm, double* rout, PcgState* st) {
  k_true_residual<VL><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, S.l_ptr.p, S.l_idx.p, S.l_v64.p, x, bm, rout, st,
                                                          S.partials.p);
}

// The body of one PCG iteration on vectors of type T.
template <typename T>
void enqueue_pcg_iteration(cudaStream_t s, const SolverImpl& S, T* r, T* sv, T* y, T* p, T* q, T* x3, double eps,
                           LoopCtl ctl) {
  const TypedArrays<T> A = arrays_of<T>(S);
  ACG_VL_SWITCH(S.vl_spmv, spmv_pq_vl, s, S, A, p, q, S.st, eps, ctl);
  const int vs = vstride<T>(S);
  k_update<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, x3, p, q, r, sv, y, S.st, S.partials.p, ctl, vs);
  enqueue_sweeps<T>(s, S, r, sv, y, S.st);
  k_ysum<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, y, S.st, S.partials.p, ctl, vs);
  k_zdot<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, y, r, p, S.st, S.partials.p, eps, 0, ctl, vs);
  k_pupdate<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, y, p, S.st, vs);
}

// ---- graph construction -----------------------------------------------------

// Current leaf nodes of a capture in progress.
std::vector<cudaGraphNode_t> capture_leaves(cudaStream_t s) {
  cudaStreamCaptureStatus status;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  ACG_CUDA(cudaStreamGetCaptureInfo(s, &status, nullptr, nullptr, &deps, &ndeps));
  return std::vector<cudaGraphNode_t>(deps, deps + ndeps);
}

cudaGraphNode_t add_while(cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, cudaGraphConditionalHandle h,
                          cudaGraph_t* body) {
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  ACG_CUDA(cudaGraphAddNode(&node, g, deps.empty() ? nullptr : deps.data(), deps.size(), &cp));
  *body = cp.conditional.phGraph_out[0];
  return node;
}

void begin_into(cudaStream_t s, cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps) {
  ACG_CUDA(cudaStreamBeginCaptureToGraph(s, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                         cudaStreamCaptureModeThreadLocal));
}
void end_into(cudaStream_t s) {
  cudaGraph_t g;
  ACG_CUDA(cudaStreamEndCapture(s, &g));
}

// Plain FP64 PCG, the reference algorithm end to end.
cudaGraphExec_t build_fp64_graph(SolverImpl& S) {
  cudaStream_t s = S.stream;
  const int n = S.n;
  cudaGraph_t top;
  ACG_CUDA(cudaGraphCreate(&top, 0));
  cudaGraphConditionalHandle h;
  ACG_CUDA(cudaGraphConditionalHandleCreate(&h, top, 1u, cudaGraphCondAssignDefault));
  LoopCtl ctl{h, 1};

  begin_into(s, top, {});
  k_gather_in<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, S.b_ext.p, S.bm.p, S.st, S.partials.p);
  k_center<double><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.bm.p, S.r64.p, S.x3_64.p, S.s64.p, S.y64.p, S.st,
                                                      S.partials.p, ctl, S.vs64);
  enqueue_sweeps<double>(s, S, S.r64.p, S.s64.p, S.y64.p, S.st);
  k_ysum<double><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.y64.p, S.st, S.partials.p, ctl, S.vs64);
  k_zdot<double><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.y64.p, S.r64.p, S.p64.p, S.st, S.partials.p, kEps64, 1, ctl,
                                                   S.vs64);
  std::vector<cudaGraphNode_t> leaves = capture_leaves(s);
  end_into(s);

  cudaGraph_t body;
  cudaGraphNode_t wnode = add_while(top, leaves, h, &body);
  begin_into(s, body, {});
  enqueue_pcg_iteration<double>(s, S, S.r64.p, S.s64.p, S.y64.p, S.p64.p, S.q64.p, S.x3_64.p, kEps64, ctl);
  end_into(s);

  begin_into(s, top, {wnode});
  k_take_best<double><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.x3_64.p, S.xf.p, S.st);
  {
    using T = double;
    ACG_VL_SWITCH(S.vl_spmv, true_res_vl, s, S, S.xf.p, S.bm.p, nullptr, S.st);
  }
  k_scatter_out<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, S.xf.p, S.x_ext.p);
  end_into(s);

  cudaGraphExec_t exec;
  ACG_CUDA(cudaGraphInstantiate(&exec, top, 0));
  cudaGraphDestroy(top);
  return exec;
}

// FP32 PCG (SpMV, sweeps, vectors) inside FP64 iterative refinement.
cudaGraphExec_t build_mixed_graph(SolverImpl& S) {
  cudaStream_t s = S.stream;
  const int n = S.n;
  const double eps32 = 1.1920928955078125e-07;
  cudaGraph_t top;
  ACG_CUDA(cudaGraphCreate(&top, 0));
  cudaGraphConditionalHandle ho;
  ACG_CUDA(cudaGraphConditionalHandleCreate(&ho, top, 1u, cudaGraphCondAssignDefault));
  LoopCtl octl{ho, 1};

  begin_into(s, top, {});
  k_gather_in<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, S.b_ext.p, S.bm.p, S.st, S.partials.p);
  // r64 = bm, x64 (xf) = 0
  k_center<double><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.bm.p, S.r64.p, S.xf.p, (double*)nullptr,
                                                      (double*)nullptr, S.st, S.partials.p, octl, 1);
  std::vector<cudaGraphNode_t> leaves = capture_leaves(s);
  end_into(s);

  cudaGraph_t obody;
  cudaGraphNode_t onode = add_while(top, leaves, ho, &obody);
  cudaGraphConditionalHandle hi;
  ACG_CUDA(cudaGraphConditionalHandleCreate(&hi, obody, 1u, cudaGraphCondAssignDefault));
  LoopCtl ictl{hi, 1};

  begin_into(s, obody, {});
  k_outer_prep<float><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.r64.p, S.r32.p, S.x3_32.p, S.s32.p, S.y32.p, S.st,
                                                         S.partials.p, ictl, S.vs32);
  enqueue_sweeps<float>(s, S, S.r32.p, S.s32.p, S.y32.p, S.st);
  k_ysum<float><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.y32.p, S.st, S.partials.p, ictl, S.vs32);
  k_zdot<float><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.y32.p, S.r32.p, S.p32.p, S.st, S.partials.p, eps32, 2, ictl,
                                                  S.vs32);
  std::vector<cudaGraphNode_t> ol = capture_leaves(s);
  end_into(s);

  cudaGraph_t ibody;
  cudaGraphNode_t inode = add_while(obody, ol, hi, &ibody);
  begin_into(s, ibody, {});
  enqueue_pcg_iteration<float>(s, S, S.r32.p, S.s32.p, S.y32.p, S.p32.p, S.q32.p, S.x3_32.p, eps32, ictl);
  end_into(s);

  begin_into(s, obody, {inode});
  k_outer_correct<float><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.x3_32.p, S.xf.p, S.st);
  {
    using T = double;
    ACG_VL_SWITCH(S.vl_spmv, true_res_vl, s, S, S.xf.p, S.bm.p, S.r64.p, S.st);
  }
  k_outer_decide<<<1, 32, 0, s>>>(S.st, octl);
  end_into(s);

  begin_into(s, top, {onode});
  k_scatter_out<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, S.xf.p, S.x_ext.p);
  end_into(s);

  cudaGraphExec_t exec;
  ACG_CUDA(cudaGraphInstantiate(&exec, top, 0));
  cudaGraphDestroy(top);
  return exec;
}

}  // namespace
}  // namespace acg

// ============================================================================
// Upload: validate the factor, level-schedule it, build device structures.
// ============================================================================
namespace acg {
namespace {

template <typename T>
std::vector<float> to_f32(const std::vector<T>& v) {
  std::vector<float> o(v.size());
  for (size_t i = 0; i < v.size(); ++i) o[i] = (float)v[i];
  return o;
}

// Host-side checks of acg_create's inputs, run before any device work (so a
// malformed factor is rejected with ACG_ERR_INVALID even where no GPU is
// present): sizes and index bases; the adjacency's structure and weights
// (finite, non-negative, no diagonal entries); the factor's structure (col a
// set of distinct vertices, non-empty columns, colptr ending at F, rowval
// naming only vertices eliminated later, i.e. an elimination order, and never
// linking two graphs of a group); fval in [0, 1]; d finite and non-negative.
// build_solver repeats the checks it depends on while it builds.
void validate_inputs(int64_t n64, const int64_t* a_colptr, const int64_t* a_rowval, const double* a_nzval,
                     const int64_t* col, int64_t ncol64, const int64_t* colptr, const int64_t* rowval,
                     const double* fval, const double* d, int64_t F, int base, int64_t nseg,
                     const int64_t* seg_off) {
  if (n64 < 2 || n64 >= (int64_t)INT32_MAX) throw InputError("n must be in [2, 2^31-1)");
  if (base != 0 && base != 1) throw InputError("index_base must be 0 or 1");
  const int64_t n = n64;
  if (nseg < 1 || nseg > n) throw InputError("graph count out of range");
  if (ncol64 < 1 || ncol64 > n - 1) throw InputError("factor column count out of range");
  std::vector<int> seg_of(n, 0);
  if (seg_off) {
    if (seg_off[0] != 0 || seg_off[nseg] != n64) throw InputError("graph offsets must start at 0 and end at n");
    for (int64_t g = 0; g < nseg; ++g) {
      if (seg_off[g + 1] - seg_off[g] < 2) throw InputError("every graph of a group needs at least 2 vertices");
      for (int64_t v = seg_off[g]; v < seg_off[g + 1]; ++v) seg_of[v] = (int)g;
    }
  }
  const int64_t abase = a_colptr[0];
  if (abase != 0 && abase != 1) throw InputError("adjacency colptr[0] must be 0 or 1");
  const int64_t m = a_colptr[n] - abase;
  if (m < 0 || m + n >= (int64_t)INT32_MAX) throw InputError("adjacency too large for 32-bit indices");
  for (int64_t c = 0; c < n; ++c) {
    if (a_colptr[c + 1] < a_colptr[c]) throw InputError("adjacency colptr not monotone");
    for (int64_t k = a_colptr[c] - abase; k < a_colptr[c + 1] - abase; ++k) {
      const int64_t r = a_rowval[k] - abase;
      if (r < 0 || r >= n) throw InputError("adjacency row index out of range");
      if (r == c) throw InputError("adjacency matrix has a diagonal entry");
      const double w = a_nzval[k];
      if (!(w >= 0.0) || std::isinf(w)) throw InputError("Adjacency matrix can not have negative edge weights");
    }
  }
  if (F < ncol64 || F >= (int64_t)INT32_MAX) throw InputError("factor size F out of range");
  std::vector<int64_t> step(n, -1);
  for (int64_t ii = 0; ii < ncol64; ++ii) {
    const int64_t u = col[ii] - base;
    if (u < 0 || u >= n) throw InputError("ldli.col entry out of range");
    if (step[u] != -1) throw InputError("ldli.col repeats a vertex");
    step[u] = ii;
  }
  for (int64_t v = 0; v < n; ++v)
    if (step[v] == -1) step[v] = ncol64;  // roots come after every eliminated column
  if (colptr[0] - base != 0) throw InputError("ldli.colptr[1] must point at the first entry");
  for (int64_t ii = 0; ii < ncol64; ++ii)
    if (colptr[ii + 1] <= colptr[ii]) throw InputError("ldli column " + std::to_string(ii + 1) + " is empty");
  if (colptr[ncol64] - base != F) throw InputError("ldli.colptr[end] must equal F+1 (1-based)");
  for (int64_t ii = 0; ii < ncol64; ++ii) {
    const int64_t u = col[ii] - base;
    for (int64_t e = colptr[ii] - base; e < colptr[ii + 1] - base; ++e) {
      const int64_t j = rowval[e] - base;
      if (j < 0 || j >= n) throw InputError("ldli.rowval entry out of range");
      if (step[j] <= ii) throw InputError("ldli.rowval names a vertex eliminated earlier (not an elimination order)");
      if (seg_of[j] != seg_of[u]) throw InputError("a factor column links two different graphs of the group");
      const double f = fval[e];
      if (!(f >= 0.0 && f <= 1.0)) throw InputError("ldli.fval entries must lie in [0, 1]");
    }
  }
  for (int64_t v = 0; v < n; ++v)
    if (!(d[v] >= 0.0) || std::isinf(d[v])) throw InputError("ldli.d must be finite and non-negative");
}

// Builds the device solver for one graph, or for the block-diagonal union of
// several graphs (seg_off: G+1 vertex offsets of contiguous diagonal blocks,
// null for one graph).  The factor has ncol eliminated columns; the vertices
// it never eliminates (one per connected block) are the roots, with d = 0.
void build_solver(SolverImpl& S, int64_t n64, const int64_t* a_colptr, const int64_t* a_rowval, const double* a_nzval,
                  const int64_t* col, int64_t ncol64, const int64_t* colptr, const int64_t* rowval,
                  const double* fval, const double* d, int64_t F, int base, const acg_options* opts,
                  int64_t nseg = 1, const int64_t* seg_off = nullptr) {
  if (n64 < 2 || n64 >= (int64_t)INT32_MAX) throw InputError("n must be in [2, 2^31-1)");
  if (base != 0 && base != 1) throw InputError("index_base must be 0 or 1");
  const int n = (int)n64;
  S.n = n;
  if (nseg < 1 || nseg > n) throw InputError("graph count out of range");
  if (ncol64 < 1 || ncol64 > n - 1) throw InputError("factor column count out of range");
  const int ncol = (int)ncol64;
  // ---- segments (graphs of a group)
  std::vector<int> seg_of(n, 0);
  S.seg_off.assign(2, 0);
  S.seg_off[1] = n;
  if (seg_off) {
    if (seg_off[0] != 0 || seg_off[nseg] != n64) throw InputError("graph offsets must start at 0 and end at n");
    S.seg_off.assign(nseg + 1, 0);
    for (int64_t g = 0; g < nseg; ++g) {
      if (seg_off[g + 1] - seg_off[g] < 2) throw InputError("every graph of a group needs at least 2 vertices");
      S.seg_off[g + 1] = (int)seg_off[g + 1];
      for (int64_t v = seg_off[g]; v < seg_off[g + 1]; ++v) seg_of[v] = (int)g;
    }
  }
  S.nseg = (int)nseg;
  // ---- adjacency
  const int64_t abase = a_colptr[0];
  if (abase != 0 && abase != 1) throw InputError("adjacency colptr[0] must be 0 or 1");
  const int64_t m = a_colptr[n] - abase;
  if (m < 0 || m + n >= (int64_t)INT32_MAX) throw InputError("adjacency too large for 32-bit indices");
  for (int c = 0; c < n; ++c)
    if (a_colptr[c + 1] < a_colptr[c]) throw InputError("adjacency colptr not monotone");
  // ---- factor validation
  if (F < ncol || F >= (int64_t)INT32_MAX) throw InputError("factor size F out of range");
  std::vector<int> step(n, -1);
  for (int ii = 0; ii < ncol; ++ii) {
    int64_t u = col[ii] - base;
    if (u < 0 || u >= n) throw InputError("ldli.col entry out of range");
    if (step[u] != -1) throw InputError("ldli.col repeats a vertex");
    step[u] = ii;
  }
  std::vector<int> roots;
  for (int v = 0; v < n; ++v)
    if (step[v] == -1) {
      step[v] = ncol + (int)roots.size();
      roots.push_back(v);
    }
  if (colptr[0] - base != 0) throw InputError("ldli.colptr[1] must point at the first entry");
  for (int ii = 0; ii < ncol; ++ii)
    if (colptr[ii + 1] <= colptr[ii]) throw InputError("ldli column " + std::to_string(ii + 1) + " is empty");
  if (colptr[ncol] - base != F) throw InputError("ldli.colptr[end] must equal F+1 (1-based)");
  // ---- levels
  std::vector<int> lev(n, 0);
  for (int ii = 0; ii < ncol; ++ii) {
    const int u = (int)(col[ii] - base);
    for (int64_t e = colptr[ii] - base; e < colptr[ii + 1] - base; ++e) {
      const int64_t j = rowval[e] - base;
      if (j < 0 || j >= n) throw InputError("ldli.rowval entry out of range");
      if (step[j] <= ii) throw InputError("ldli.rowval names a vertex eliminated earlier (not an elimination order)");
      if (seg_of[j] != seg_of[u]) throw InputError("a factor column links two different graphs of the group");
      const double f = fval[e];
      if (!(f >= 0.0 && f <= 1.0)) throw InputError("ldli.fval entries must lie in [0, 1]");
      if (lev[j] < lev[u] + 1) lev[j] = lev[u] + 1;
    }
  }
  for (int v = 0; v < n; ++v)
    if (!(d[v] >= 0.0) || std::isinf(d[v])) throw InputError("ldli.d must be finite and non-negative");
  int nlev = 0;
  for (int v = 0; v < n; ++v) nlev = std::max(nlev, lev[v] + 1);
  S.nlev = nlev;
  // Internal order: by graph, then level; inside a level by decreasing
  // forward in-degree (then elimination step), so heavy vertices come first.
  std::vector<int> indeg(n, 0);
  for (int64_t e = 0; e < F; ++e) indeg[rowval[e] - base]++;
  std::vector<int> perm(n), e2i(n);
  for (int v = 0; v < n; ++v) perm[v] = v;
  const bool by_id = opts && opts->level_order == 1;
  std::sort(perm.begin(), perm.end(), [&](int x, int y) {
    if (seg_of[x] != seg_of[y]) return seg_of[x] < seg_of[y];
    if (lev[x] != lev[y]) return lev[x] < lev[y];
    if (by_id) return x < y;
    if (indeg[x] != indeg[y]) return indeg[x] > indeg[y];
    return step[x] < step[y];
  });
  for (int i = 0; i < n; ++i) e2i[perm[i]] = i;
  // level runs: runs[l] = list of {first, last+1} internal ranges of level l (one per graph)
  std::vector<std::vector<std::pair<int, int>>> runs(nlev);
  for (int i = 0; i < n;) {
    int j = i;
    while (j < n && seg_of[perm[j]] == seg_of[perm[i]] && lev[perm[j]] == lev[perm[i]]) ++j;
    runs[lev[perm[i]]].emplace_back(i, j);
    i = j;
  }
  // global level offsets (meaningful for one graph: its levels are contiguous)
  S.lvl_off.assign(nlev + 1, 0);
  for (int v = 0; v < n; ++v) S.lvl_off[lev[v] + 1]++;
  for (int l = 0; l < nlev; ++l) S.lvl_off[l + 1] += S.lvl_off[l];
  S.heavy.assign(nlev, 0);
  for (int v = 0; v < n; ++v)
    if (indeg[v] > 32) S.heavy[lev[v]]++;
  // ---- folded coefficients
  std::vector<double> coef(F);
  std::vector<double> g(n, 1.0);
  for (int ii = 0; ii < ncol; ++ii) {
    const int u = (int)(col[ii] - base);
    const int64_t j0 = colptr[ii] - base, j1 = colptr[ii + 1] - base - 1;
    double prod = 1.0;
    for (int64_t e = j0; e < j1; ++e) {
      coef[e] = fval[e] * prod;
      prod = prod * (1.0 - fval[e]);
    }
    coef[j1] = prod;
    g[u] = d[u] != 0.0 ? prod * prod / d[u] : prod * prod;
  }
  // forward: in-edges by internal target, in elimination order of the source
  std::vector<int> fptr(n + 1, 0), fidx(F);
  std::vector<double> fc(F);
  for (int64_t e = 0; e < F; ++e) fptr[e2i[rowval[e] - base] + 1]++;
  for (int v = 0; v < n; ++v) fptr[v + 1] += fptr[v];
  {
    std::vector<int> pos(fptr.begin(), fptr.end() - 1);
    for (int ii = 0; ii < ncol; ++ii) {
      const int us = e2i[col[ii] - base];
      for (int64_t e = colptr[ii] - base; e < colptr[ii + 1] - base; ++e) {
        const int t = e2i[rowval[e] - base];
        fidx[pos[t]] = us;
        fc[pos[t]] = coef[e];
        pos[t]++;
      }
    }
  }
  // backward: column entries by internal source
  std::vector<int> bptr(n + 1, 0), bidx(F);
  std::vector<double> bc(F), gi(n);
  for (int v = 0; v < n; ++v) {
    const int u = perm[v];
    gi[v] = g[u];
    bptr[v + 1] = bptr[v];
    if (step[u] >= ncol) continue;  // a root: no column
    const int ii = step[u];
    for (int64_t e = colptr[ii] - base; e < colptr[ii + 1] - base; ++e) {
      bidx[bptr[v + 1]] = e2i[rowval[e] - base];
      bc[bptr[v + 1]] = coef[e];
      bptr[v + 1]++;
    }
  }
  // Entries of a vertex in the order their values become ready: the sweeps
  // walk a long row in rounds, and the input finished last (forward: the
  // highest internal index; backward: the lowest) belongs in the last round
  // so the earlier rounds overlap the wait for it.
  {
    std::vector<std::pair<int, double>> tmp;
    auto order = [&](std::vector<int>& ptr, std::vector<int>& ix, std::vector<double>& cv, bool descending) {
      for (int v = 0; v < n; ++v) {
        tmp.clear();
        for (int k = ptr[v]; k < ptr[v + 1]; ++k) tmp.emplace_back(ix[k], cv[k]);
        if (descending)
          std::stable_sort(tmp.begin(), tmp.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        else
          std::stable_sort(tmp.begin(), tmp.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        for (int k = ptr[v]; k < ptr[v + 1]; ++k) {
          ix[k] = tmp[k - ptr[v]].first;
          cv[k] = tmp[k - ptr[v]].second;
        }
      }
    };
    order(fptr, fidx, fc, false);
    order(bptr, bidx, bc, true);
  }
  // ---- dense tail: the final levels as one dense triangular block (one
  // graph, sync-free sweeps; the per-level engine and the one-CTA tail keep
  // the full entry lists)
  S.dt_K = 0;
  if (nseg == 1 && !(opts && (opts->sweep_lanes == 1 || opts->tail == 2 || opts->dense_tail < 0))) {
    int kmax = (opts && opts->dense_tail > 0) ? opts->dense_tail : kDenseDefaultK;
    kmax = std::min(std::min(kmax, kDenseMaxK), n / 4);
    int L0 = nlev;
    while (L0 > 0 && n - S.lvl_off[L0 - 1] <= kmax) --L0;
    if (nlev - L0 >= kDenseMinLevels && n - S.lvl_off[L0] > 0) {
      S.dt_L0 = L0;
      S.dt_v0 = S.lvl_off[L0];
      S.dt_K = n - S.dt_v0;
    }
  }
  std::vector<double> dense_m;
  if (S.dt_K) {
    const int K = S.dt_K, v0 = S.dt_v0;
    // M = (I - C_TT)^{-1}, row by row: M[i,:] = e_i + sum over tail inputs u of
    // i of coef * M[u,:] (inputs precede i in internal order).  Threads own
    // interleaved blocks of 64 columns and walk all rows, so no thread waits
    // for another and each entry is summed in one fixed order.
    dense_m.assign((size_t)K * K, 0.0);
    const int nthreads = std::max(1, std::min(32, (int)std::thread::hardware_concurrency()));
    auto work = [&](int tid) {
      for (int i = 0; i < K; ++i) {
        double* row = &dense_m[(size_t)i * K];
        for (int cb = tid * 64; cb <= i; cb += nthreads * 64) {
          const int ce = std::min(cb + 64, i + 1);
          if (i >= cb && i < ce) row[i] = 1.0;
          for (int k = fptr[v0 + i]; k < fptr[v0 + i + 1]; ++k) {
            const int u = fidx[k] - v0;
            if (u < 0) continue;
            const double c = fc[k];
            const double* mu = &dense_m[(size_t)u * K];
            const int e2 = std::min(ce, u + 1);
            for (int j = cb; j < e2; ++j) row[j] += c * mu[j];
          }
        }
      }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& t : pool) t.join();
    // the sweep keeps only the head inputs of tail vertices (a prefix: entries
    // are in increasing internal order)
    std::vector<int> nptr(n + 1, 0);
    int w = 0;
    for (int v = 0; v < n; ++v) {
      const int k0 = fptr[v], k1 = fptr[v + 1];
      nptr[v] = w;
      for (int k = k0; k < k1; ++k) {
        if (v >= v0 && fidx[k] >= v0) break;
        fidx[w] = fidx[k];
        fc[w] = fc[k];
        ++w;
      }
    }
    nptr[n] = w;
    fptr.swap(nptr);
    fidx.resize(w);
    fc.resize(w);
  }
  // Laplacian rows in internal order; diagonal = a*ones summed in column order
  std::vector<int> lptr(n + 1, 0), lidx(m + n);
  std::vector<double> lv(m + n);
  {
    std::vector<std::pair<int, double>> row;
    for (int i = 0; i < n; ++i) {
      const int u = perm[i];
      row.clear();
      double deg = 0.0;
      for (int64_t k = a_colptr[u] - abase; k < a_colptr[u + 1] - abase; ++k) {
        const int64_t c = a_rowval[k] - abase;
        if (c < 0 || c >= n) throw InputError("adjacency row index out of range");
        if (c == u) throw InputError("adjacency matrix has a diagonal entry");
        const double w = a_nzval[k];
        if (!(w >= 0.0) || std::isinf(w)) throw InputError("Adjacency matrix can not have negative edge weights");
        deg += w;
        row.emplace_back(e2i[c], 0.0 - w);
      }
      row.emplace_back(i, deg);
      std::sort(row.begin(), row.end(),
                [](const std::pair<int, double>& x, const std::pair<int, double>& y) { return x.first < y.first; });
      lptr[i + 1] = lptr[i] + (int)row.size();
      for (size_t k = 0; k < row.size(); ++k) {
        lidx[lptr[i] + k] = row[k].first;
        lv[lptr[i] + k] = row[k].second;
      }
    }
  }
  S.nnz_l = m + n;
  S.nnz_f = F;
  // ---- tuning knobs
  S.vl_spmv = choose_vl((double)(m + n) / n);
  S.thin_max_width = 2048;
  if (opts) {
    if (opts->spmv_lanes > 0) S.vl_spmv = opts->spmv_lanes;
    if (opts->wide_level_min > 0) S.thin_max_width = opts->wide_level_min;
  }
  if (S.vl_spmv != 2 && S.vl_spmv != 4 && S.vl_spmv != 8 && S.vl_spmv != 16)
    throw InputError("lane counts must be 2, 4, 8 or 16");
  // ---- sweep plans: runs of consecutive levels narrower than thin_max_width
  // whose values fit in shared memory go to one CTA; other levels get a
  // grid launch each.
  {
    int optin = 0;
    ACG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, S.device));
    S.smem_optin = (size_t)optin;
  }
  const size_t smem_cap = S.smem_optin > 4096 ? S.smem_optin - 2048 : 0;
  for (int pi = 0; pi < 2; ++pi) {
    auto& plan = S.plan[pi];
    plan.clear();
    auto bytes = [&](int nv, int nl) {
      return pi == 0 ? thin_smem_bytes<double>(nv, nl) : thin_smem_bytes<float>(nv, nl);
    };
    for (int l = 0; l < nlev;) {
      const int w = S.lvl_off[l + 1] - S.lvl_off[l];
      if (w >= S.thin_max_width || bytes(w, 1) > smem_cap) {
        plan.push_back({0, l, l + 1, S.lvl_off[l], S.lvl_off[l + 1], S.heavy[l], 0});
        ++l;
        continue;
      }
      int l1 = l;
      while (l1 < nlev && S.lvl_off[l1 + 1] - S.lvl_off[l1] < S.thin_max_width &&
             bytes(S.lvl_off[l1 + 1] - S.lvl_off[l], l1 + 1 - l) <= smem_cap)
        ++l1;
      plan.push_back({1, l, l1, S.lvl_off[l], S.lvl_off[l1], 0, bytes(S.lvl_off[l1] - S.lvl_off[l], l1 - l)});
      l = l1;
    }
  }
  // ---- sync-free task tables: tasks in level order (backward: reverse level
  // order); a vertex with more than sweep_heavy entries (default 16) is a
  // task of its own on a whole warp, other vertices go four to a task within
  // one level.
  {
    std::vector<int> outdeg(n, 0);
    for (int v = 0; v < n; ++v) outdeg[v] = bptr[v + 1] - bptr[v];
    auto emit_level = [](std::vector<SweepTask>& tasks, int vs, int ve, const std::vector<int>& deg,
                         const std::vector<int>& ptr, int heavy_min) {
      int run = -1, cnt = 0;
      auto push = [&](int v, int c, int heavy) {
        SweepTask t = {};
        t.v = v;
        t.cnt_heavy = (c << 1) | heavy;
        for (int i = 0; i <= c; ++i) t.p[i] = ptr[v + i];
        tasks.push_back(t);
      };
      auto flush = [&]() {
        if (cnt) push(run, cnt, 0);
        cnt = 0;
      };
      for (int v = vs; v < ve; ++v) {
        if (deg[v] > heavy_min) {
          flush();
          push(v, 1, 1);
          continue;
        }
        if (cnt == 0) run = v;
        if (++cnt == 4) flush();
      }
      flush();
    };
    std::vector<int> fdeg(n);
    for (int v = 0; v < n; ++v) fdeg[v] = fptr[v + 1] - fptr[v];
    const int sheavy = (opts && opts->sweep_heavy > 0) ? opts->sweep_heavy : 16;
    std::vector<SweepTask> tf, tb;
    std::vector<int2> lf(nlev), lb(nlev);  // {first task, count} per level
    for (int l = 0; l < nlev; ++l) {
      const int t0 = (int)tf.size();
      for (const auto& r : runs[l]) emit_level(tf, r.first, r.second, fdeg, fptr, sheavy);
      lf[l] = make_int2(t0, (int)tf.size() - t0);
    }
    const int blev = S.dt_K ? S.dt_L0 : nlev;  // levels the backward sweep walks
    for (int l = nlev - 1; l >= blev; --l) lb[l] = make_int2((int)tb.size(), 0);
    for (int l = blev - 1; l >= 0; --l) {
      const int t0 = (int)tb.size();
      for (const auto& r : runs[l]) emit_level(tb, r.first, r.second, outdeg, bptr, sheavy);
      lb[l] = make_int2(t0, (int)tb.size() - t0);
    }
    // the tail: the longest run of final levels with at most 32 tasks in both
    // tables whose values fit in shared memory (FP64 sizes, so both precisions fit)
    {
      int optin = 0;
      ACG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, S.device));
      const size_t cap = optin > 8192 ? (size_t)optin - 4096 : 0;
      int lt = nlev, nv = 0;
      while (lt > 0) {
        const int l = lt - 1;
        const int w = S.lvl_off[l + 1] - S.lvl_off[l];
        if (lf[l].y > kTailWarps || lb[l].y > kTailWarps) break;
        if (tail_smem_bytes<double>(nv + w, nlev - l) > cap) break;
        nv += w;
        lt = l;
      }
      if (nlev - lt >= 8 && nseg == 1 && opts && opts->tail == 2) {
        S.tail_nl = nlev - lt;
        S.tail_v0 = S.lvl_off[lt];
        S.tail_nv = n - S.tail_v0;
        S.tail_tf0 = lf[lt].x;
        S.tail_tb0 = lb[lt].x + lb[lt].y;
        std::vector<int2> tlf(lf.begin() + lt, lf.end()), tlb(lb.begin() + lt, lb.end());
        S.tail_lvl_f.upload(tlf, S.stream);
        S.tail_lvl_b.upload(tlb, S.stream);
        const int tb_bytes = (int)tail_smem_bytes<double>(S.tail_nv, S.tail_nl);
        ACG_CUDA(cudaFuncSetAttribute(k_tail<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tb_bytes));
        ACG_CUDA(cudaFuncSetAttribute(k_tail<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tb_bytes));
        ACG_CUDA(cudaFuncSetAttribute(k_tail<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tb_bytes));
        ACG_CUDA(cudaFuncSetAttribute(k_tail<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tb_bytes));
      } else {
        S.tail_nl = 0;
      }
    }
    // task tables of the batched sweeps: a vertex with more than bheavy
    // (backward) or fheavy (forward) entries gets a whole warp
    {
      const int bheavy = (opts && opts->batch_bwd_heavy > 0) ? opts->batch_bwd_heavy : 8;
      const int fheavy = (opts && opts->batch_fwd_heavy > 0) ? opts->batch_fwd_heavy : 8;
      std::vector<SweepTask> tbb, tfb;
      S.tbb_from.assign(nlev, 0);
      S.tfb_upto.assign(nlev, 0);
      for (int l = blev - 1; l >= 0; --l) {
        for (const auto& r : runs[l]) emit_level(tbb, r.first, r.second, outdeg, bptr, bheavy);
        S.tbb_from[l] = (int)tbb.size();
      }
      for (int l = 0; l < nlev; ++l) {
        for (const auto& r : runs[l]) emit_level(tfb, r.first, r.second, fdeg, fptr, fheavy);
        S.tfb_upto[l] = (int)tfb.size();
      }
      // Testing only: blank one forward task record (it stores nothing), so
      // the values of its vertices are never produced and the waits on them
      // run out after spin_limit polls; the solve then reports
      // ACG_ERR_TIMEOUT.  This is how the bounded waits are tested without
      // faulting or hanging the GPU.
      const int blank = opts ? opts->test_unproduced_task : 0;
      if (blank > 0) {
        if (blank > (int)tf.size() || blank > (int)tfb.size())
          throw InputError("test_unproduced_task is beyond the forward task tables");
        tf[blank - 1].cnt_heavy = 0;
        tfb[blank - 1].cnt_heavy = 0;
      }
      S.ntasks_bb = (int)tbb.size();
      S.tasks_bb.upload(tbb, S.stream);
      S.ntasks_fb = (int)tfb.size();
      S.tasks_fb.upload(tfb, S.stream);
    }
    S.ntasks_f = (int)tf.size();
    S.ntasks_b = (int)tb.size();
    S.nnz_fsweep = fptr[n];
    S.nnz_bsweep = bptr[S.dt_K ? S.dt_v0 : n];
    S.tasks_f.upload(tf, S.stream);
    S.tasks_b.upload(tb, S.stream);
    int sms = 0;
    ACG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S.device));
    int occ[4] = {0, 0, 0, 0};
    ACG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], k_sweep<double, true>, kSweepThreads, 0));
    ACG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], k_sweep<double, false>, kSweepThreads, 0));
    ACG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], k_sweep<float, true>, kSweepThreads, 0));
    ACG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[3], k_sweep<float, false>, kSweepThreads, 0));
    // Resident blocks (8 warps each) per SM: a deep, narrow DAG gains nothing
    // from more warps (they add polling traffic without shortening the chains),
    // a wide one is throughput-bound in its wide levels and gains from them.
    // Automatic choice by the tasks per swept level (measured: the 2M
    // path+matchings graph, ~150 per level, is fastest with 1; the 1M 3D grid,
    // ~750, with 2; 256 graphs in one launch, thousands, with 4).
    int cap = 1;
    if (opts && opts->sweep_blocks_per_sm > 0) {
      cap = opts->sweep_blocks_per_sm;
    } else {
      const int swept = std::max(1, (S.dt_K ? S.dt_L0 : nlev));
      const double per_level = (double)std::max(S.ntasks_f, S.ntasks_b) / swept;
      cap = per_level < 300.0 ? 1 : (per_level < 2000.0 ? 2 : 4);
    }
    S.sweep_blocks[0] = sms * std::max(1, std::min(cap, std::min(occ[0], occ[1])));
    S.sweep_blocks[1] = sms * std::max(1, std::min(cap, std::min(occ[2], occ[3])));
    S.sweep_mode = (opts && opts->sweep_lanes == 1 && nseg == 1) ? 1 : 0;
    if (opts && opts->poll_mode > 0) S.poll_mode = opts->poll_mode - 1;
    if (opts && opts->spin_limit > 0) S.spin_limit = (unsigned)opts->spin_limit;
    if (opts && opts->min_inner_tol > 0) S.min_inner_tol = std::min(0.25, opts->min_inner_tol);
    S.batch_bps = (opts && opts->batch_blocks_per_sm > 0) ? opts->batch_blocks_per_sm : 0;
  }
  ACG_CUDA(cudaFuncSetAttribute(k_thin<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
  ACG_CUDA(cudaFuncSetAttribute(k_thin<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
  ACG_CUDA(cudaFuncSetAttribute(k_thin<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
  ACG_CUDA(cudaFuncSetAttribute(k_thin<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
  // ---- upload
  cudaStream_t s = S.stream;
  S.perm.upload(perm, s);
  {
    std::vector<int> iperm(perm.size());
    for (size_t v = 0; v < perm.size(); ++v) iperm[perm[v]] = (int)v;
    S.iperm.upload(iperm, s);
  }
  S.lvl_off_d.upload(S.lvl_off, s);
  S.l_ptr.upload(lptr, s);
  S.l_idx.upload(lidx, s);
  S.l_v64.upload(lv, s);
  S.l_v32.upload(to_f32(lv), s);
  S.f_ptr.upload(fptr, s);
  S.f_idx.upload(fidx, s);
  S.f_c64.upload(fc, s);
  S.f_c32.upload(to_f32(fc), s);
  S.b_ptr.upload(bptr, s);
  S.b_idx.upload(bidx, s);
  S.b_c64.upload(bc, s);
  S.b_c32.upload(to_f32(bc), s);
  S.g64.upload(gi, s);
  S.g32.upload(to_f32(gi), s);
  if (S.dt_K) {
    S.dt_M64.upload(dense_m, s);
    S.dt_M32.upload(to_f32(dense_m), s);
    // partial tiles for up to kMaxBatch columns, so no later growth moves them
    S.dt_part_cols = kMaxBatch;
    S.dt_part.alloc((size_t)dense_chunks(S.dt_K) * S.dt_K * kMaxBatch);
  }
  // one 32-byte sector per vertex in the sweep vectors of the sync-free engine
  // on one graph; the per-level engine and the one-CTA tail index them densely,
  // and so does the group solver, whose wide union DAG makes its vector passes
  // bandwidth-bound (measured on 256 graphs: 1,748 solves/s dense, 1,552 padded)
  const bool pad = S.sweep_mode == 0 && S.tail_nl == 0 && nseg == 1 && !(opts && opts->sweep_stride == 1);
  S.vs64 = pad ? 32 / (int)sizeof(double) : 1;
  S.vs32 = pad ? 32 / (int)sizeof(float) : 1;
  for (DevBuf<double>* b : {&S.b_ext, &S.x_ext, &S.bm, &S.r64, &S.p64, &S.q64, &S.xf}) b->alloc(n);
  for (DevBuf<double>* b : {&S.s64, &S.y64}) b->alloc((size_t)n * S.vs64);
  S.x3_64.alloc((size_t)3 * n);
  for (DevBuf<float>* b : {&S.r32, &S.p32, &S.q32}) b->alloc(n);
  for (DevBuf<float>* b : {&S.s32, &S.y32}) b->alloc((size_t)n * S.vs32);
  S.x3_32.alloc((size_t)3 * n);
  S.partials.alloc((size_t)4 * kMaxPartialBlocks);
  ACG_CUDA(cudaMalloc(&S.st, sizeof(PcgState)));
  ACG_CUDA(cudaMemsetAsync(S.st, 0, sizeof(PcgState), s));
  ACG_CUDA(cudaMallocHost(&S.h_st, sizeof(PcgState)));
  std::memset(S.h_st, 0, sizeof(PcgState));
  if (S.nseg > 1) {
    // chunks of at most kChunk vertices, each inside one graph
    std::vector<SegChunk> ch;
    std::vector<int> first(S.nseg), cnt(S.nseg);
    for (int g = 0; g < S.nseg; ++g) {
      first[g] = (int)ch.size();
      for (int a = S.seg_off[g]; a < S.seg_off[g + 1]; a += kChunk)
        ch.push_back({g, a, std::min(a + kChunk, S.seg_off[g + 1]), 0});
      cnt[g] = (int)ch.size() - first[g];
    }
    S.nchunks = (int)ch.size();
    S.chunks.upload(ch, s);
    S.seg_first.upload(first, s);
    S.seg_nchunk.upload(cnt, s);
    S.seg_cnt.alloc((size_t)8 * S.nseg);
    ACG_CUDA(cudaMemsetAsync(S.seg_cnt.p, 0, sizeof(unsigned int) * 8 * S.nseg, s));
    S.gpartials.alloc((size_t)4 * S.nchunks);
    ACG_CUDA(cudaMalloc(&S.gstates, sizeof(PcgState) * S.nseg));
    ACG_CUDA(cudaMalloc(&S.gflags, sizeof(PcgState)));
    ACG_CUDA(cudaMalloc(&S.gsh, sizeof(GroupShared)));
    ACG_CUDA(cudaMemsetAsync(S.gflags, 0, sizeof(PcgState), s));
    ACG_CUDA(cudaMemsetAsync(S.gsh, 0, sizeof(GroupShared), s));
    ACG_CUDA(cudaMallocHost(&S.h_gstates, sizeof(PcgState) * S.nseg));
  }
  ACG_CUDA(cudaStreamSynchronize(s));
}

// ---- small kernels for the one-shot entry points ---------------------------

template <typename T>
__global__ void k_cast_from64(int n, const double* __restrict__ a, T* __restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (T)a[i];
}
template <typename T>
__global__ void k_minus_mean(int n, const T* __restrict__ y, const PcgState* st, double* __restrict__ out, int vs) {
  const double mu = st->mean;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = (double)y[(size_t)i * vs] - mu;
}
template <typename T, int VL>
__global__ void __launch_bounds__(kVecThreads) k_spmv_plain(int n, const int* __restrict__ ptr, const int* __restrict__ idx,
                                                            const T* __restrict__ val, const T* __restrict__ x, double* __restrict__ y) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = gt & (VL - 1);
  const int groups = gridDim.x * blockDim.x / VL;
  for (int base = (gt & ~31) / VL; base < n; base += groups) {
    const int row = base + (gt & 31) / VL;
    const bool active = row < n;
    T s = row_dot<T, VL>(ptr, idx, val, x, row, active, lane);
    if (active && lane == 0) y[row] = (double)s;
  }
}
template <typename T, int VL>
void spmv_plain_vl(cudaStream_t s, const SolverImpl& S, const TypedArrays<T>& A, const T* x, double* y) {
  k_spmv_plain<T, VL><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, A.lp, A.li, A.lv, x, y);
}

void reset_state_for_direct_use(SolverImpl& S) {
  std::memset(S.h_st, 0, sizeof(PcgState));
  ACG_CUDA(cudaMemcpyAsync(S.st, S.h_st, sizeof(PcgState), cudaMemcpyHostToDevice, S.stream));
}

template <typename T>
void ldlsolve_impl(SolverImpl& S, T* rbuf, T* sbuf, T* ybuf) {
  cudaStream_t s = S.stream;
  const int n = S.n;
  reset_state_for_direct_use(S);
  LoopCtl none{0, 0};
  k_gather_in<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, S.b_ext.p, S.bm.p, S.st, S.partials.p);
  k_cast_from64<T><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.bm.p, rbuf);
  const int vs = vstride<T>(S);
  k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>(n, sbuf, ybuf, vs);
  enqueue_sweeps<T>(s, S, rbuf, sbuf, ybuf, S.st);
  k_ysum<T><<<kVecBlocks, kVecThreads, 0, s>>>(n, ybuf, S.st, S.partials.p, none, vs);
  k_minus_mean<T><<<kVecBlocks, kVecThreads, 0, s>>>(n, ybuf, S.st, S.xf.p, vs);
  k_scatter_out<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, S.xf.p, S.x_ext.p);
}

// ---- allocation-free LDLsolver ----------------------------------------------
//
// Some callers cannot allocate device memory at the moment they apply the
// preconditioner: a serving loop whose device memory comes from a pool that
// must not grow after start-up, a host runtime whose own allocator owns the
// GPU's memory, or a caller that cannot let cudaMalloc/cudaFree synchronize
// the device under its other streams.  For them
// acg_ldlsolve_noalloc keeps every piece of its scratch (the input in solver
// order, the forward and backward sweep vectors, the reduction partials, the
// dense tail's partial tiles and the scalar state) in the one fixed array
// below, which the library reserves on every GPU it is loaded on, for as long
// as the process lives.
constexpr int kNoAllocMaxN = ACG_NOALLOC_MAX_N;
constexpr size_t kNoAllocVec = (size_t)kNoAllocMaxN * sizeof(double);
constexpr size_t kNoAllocPartials = (size_t)4 * kMaxPartialBlocks * sizeof(double);
// a dense tail has at most min(kDenseMaxK, n / 4) vertices
constexpr int kNoAllocDenseK = kDenseMaxK < kNoAllocMaxN / 4 ? kDenseMaxK : kNoAllocMaxN / 4;
constexpr size_t kNoAllocDense = (size_t)dense_chunks(kNoAllocDenseK) * kNoAllocDenseK * sizeof(double);
constexpr size_t kNoAllocState = 4 * kNoAllocVec + kNoAllocPartials + kNoAllocDense;
constexpr size_t kNoAllocBytes = kNoAllocState + ((sizeof(PcgState) + 255) / 256) * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
unsigned char* g_noalloc_addr[256] = {};

// Device address of the scratch array on the current device.  Host code must
// not use g_noalloc_scratch itself: on the host that name is only a stand-in.
unsigned char* noalloc_scratch_for_current_device(int device) {
  if (device < 0 || device >= 256) throw InputError("device ordinal out of range for the no-alloc scratch table");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* ptr = nullptr;
    ACG_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    g_noalloc_addr[device] = static_cast<unsigned char*>(ptr);
  }
  return g_noalloc_addr[device];
}

template <typename T>
void ldlsolve_noalloc_impl(const SolverImpl& S, cudaStream_t s, const double* r_ext, double* y_ext,
                           unsigned char* base) {
  const int n = S.n;
  double* r64 = reinterpret_cast<double*>(base);
  T* rT = reinterpret_cast<T*>(base + kNoAllocVec);
  T* sv = reinterpret_cast<T*>(base + 2 * kNoAllocVec);
  T* yv = reinterpret_cast<T*>(base + 3 * kNoAllocVec);
  double* partials = reinterpret_cast<double*>(base + 4 * kNoAllocVec);
  T* dense_part = reinterpret_cast<T*>(base + 4 * kNoAllocVec + kNoAllocPartials);
  PcgState* st = reinterpret_cast<PcgState*>(base + kNoAllocState);
  LoopCtl none{0, 0};
  // the state (done flag, sweep error flag, reduction tickets) must start at zero
  ACG_CUDA(cudaMemsetAsync(st, 0, sizeof(PcgState), s));
  k_gather_in<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, r_ext, r64, st, partials);
  k_cast_from64<T><<<kVecBlocks, kVecThreads, 0, s>>>(n, r64, rT);
  // compact vectors (one value per vertex): the fixed array holds n values each
  k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>(n, sv, yv, 1);
  enqueue_sweeps<T>(s, S, rT, sv, yv, st, dense_part, 1);
  k_ysum<T><<<kVecBlocks, kVecThreads, 0, s>>>(n, yv, st, partials, none, 1);
  k_minus_mean<T><<<kVecBlocks, kVecThreads, 0, s>>>(n, yv, st, r64, 1);
  k_scatter_out<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, r64, y_ext);
}

int noalloc_sweep_error(unsigned char* base) {
  PcgState hs;
  ACG_CUDA(cudaMemcpy(&hs, base + kNoAllocState, sizeof(PcgState), cudaMemcpyDeviceToHost));
  return hs.sweep_error;
}

template <typename T>
void lapmul_impl(SolverImpl& S, T* xbuf) {
  cudaStream_t s = S.stream;
  const int n = S.n;
  reset_state_for_direct_use(S);
  k_gather_in<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, S.b_ext.p, S.bm.p, S.st, S.partials.p);
  k_cast_from64<T><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.bm.p, xbuf);
  const TypedArrays<T> A = arrays_of<T>(S);
  ACG_VL_SWITCH(S.vl_spmv, spmv_plain_vl, s, S, A, xbuf, S.xf.p);
  k_scatter_out<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, S.xf.p, S.x_ext.p);
}


// Device time per call of the solve's kernels, each captured `reps` times in a
// graph and timed with CUDA events on the solver's stream.  Sweeps are timed
// together with the kernel that marks their output pending, minus that
// kernel's own time.
template <typename T>
void time_kernels_t(SolverImpl& S, int reps, acg_kernel_times* out, T* r, T* sv, T* y, T* p, T* q) {
  cudaStream_t s = S.stream;
  reset_state_for_direct_use(S);
  ACG_CUDA(cudaStreamSynchronize(s));
  const TypedArrays<T> A = arrays_of<T>(S);
  LoopCtl none{0, 0};
  auto time_graph = [&](auto&& body) -> double {
    cudaGraph_t g;
    ACG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < reps; ++i) body();
    ACG_CUDA(cudaStreamEndCapture(s, &g));
    cudaGraphExec_t ge;
    ACG_CUDA(cudaGraphInstantiate(&ge, g, 0));
    ACG_CUDA(cudaGraphLaunch(ge, s));  // warm-up
    cudaEvent_t e0, e1;
    ACG_CUDA(cudaEventCreate(&e0));
    ACG_CUDA(cudaEventCreate(&e1));
    ACG_CUDA(cudaEventRecord(e0, s));
    ACG_CUDA(cudaGraphLaunch(ge, s));
    ACG_CUDA(cudaEventRecord(e1, s));
    ACG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    ACG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    return (double)ms / reps;
  };
  const int vs = vstride<T>(S);
  auto fill_s = [&]() { k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, sv, (T*)nullptr, vs); };
  auto fill_y = [&]() { k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, y, (T*)nullptr, vs); };
  const double t_fill = time_graph(fill_s);
  out->spmv_ms = time_graph([&]() { ACG_VL_SWITCH(S.vl_spmv, spmv_plain_vl, s, S, A, p, S.xf.p); });
  out->forward_ms = time_graph([&]() {
    fill_s();
    enqueue_forward<T>(s, S, r, sv, S.st);
  }) - t_fill;
  out->backward_ms = time_graph([&]() {
    fill_y();
    enqueue_backward<T>(s, S, sv, y, S.st);
  }) - t_fill;
  out->iteration_ms = time_graph([&]() {
    // the kernels of one PCG iteration without the stop logic taking effect
    ACG_VL_SWITCH(S.vl_spmv, spmv_plain_vl, s, S, A, p, S.xf.p);
    k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, sv, y, vs);
    enqueue_sweeps<T>(s, S, r, sv, y, S.st);
    k_ysum<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, y, S.st, S.partials.p, none, vs);
    k_ysum<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, y, S.st, S.partials.p, none, vs);
    k_pupdate<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, y, q, S.st, vs);
  });
  out->forward_sweep_ms = time_graph([&]() {
    fill_s();
    enqueue_forward<T>(s, S, r, sv, S.st, (T*)nullptr, false);
  }) - t_fill;
  // the backward sweep alone reads the tail values the dense product wrote in
  // the backward_ms runs above, so only the head is marked pending
  auto fill_yh = [&]() {
    k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>(S.dt_K ? S.dt_v0 : S.n, y, (T*)nullptr, vs);
  };
  const double t_fill_h = time_graph(fill_yh);
  out->backward_sweep_ms = time_graph([&]() {
    fill_yh();
    enqueue_backward<T>(s, S, sv, y, S.st, (T*)nullptr, false);
  }) - t_fill_h;
  out->dense_ms = S.dt_K ? time_graph([&]() {
    enqueue_dense<T, 0>(s, S, true, sv, (T*)nullptr, reinterpret_cast<T*>(S.dt_part.p), &S.st->done, vs);
    enqueue_dense<T, 0>(s, S, false, sv, y, reinterpret_cast<T*>(S.dt_part.p), &S.st->done, vs);
  }) : 0.0;
  const double vb = sizeof(T), nv = S.n;
  // mat-vec: row pointers, (index, value) per entry, x once, y (FP64) out
  out->spmv_bytes = 4.0 * (nv + 1) + (double)S.nnz_l * (4.0 + vb) + nv * vb + nv * 8.0;
  // sweeps: (index, coefficient) per entry, one 32-byte task record per task,
  // aux (r or g) in, own forward value (backward), each input value once, output
  out->forward_sweep_bytes = (double)S.nnz_fsweep * (4.0 + vb) + 32.0 * S.ntasks_f + nv * vb * 3.0;
  out->backward_sweep_bytes = (double)S.nnz_bsweep * (4.0 + vb) + 32.0 * S.ntasks_b + nv * vb * 4.0;
  // dense tail: the K(K+1)/2 entries of M once per product
  const double kk = (double)S.dt_K;
  out->dense_bytes = 2.0 * kk * (kk + 1.0) / 2.0 * vb;
  out->forward_bytes = out->forward_sweep_bytes + out->dense_bytes / 2.0;
  out->backward_bytes = out->backward_sweep_bytes + out->dense_bytes / 2.0;
  const int sweep_launches = S.sweep_mode == 0 ? 1 : (int)S.plan[plan_index<T>()].size();
  const int dense_launches = S.dt_K ? 2 : 0;
  out->launches_per_iteration = 6 + 2 * (sweep_launches + dense_launches);
  out->forward_launches = sweep_launches + dense_launches;
  ACG_CUDA(cudaStreamSynchronize(s));
  PcgState hs;
  ACG_CUDA(cudaMemcpy(&hs, S.st, sizeof(PcgState), cudaMemcpyDeviceToHost));
  if (hs.sweep_error) throw CudaError("a sync-free sweep wait gave up while timing");
}

void time_kernels(SolverImpl& S, int precision, int reps, acg_kernel_times* out) {
  if (precision == 0) time_kernels_t<double>(S, reps, out, S.r64.p, S.s64.p, S.y64.p, S.p64.p, S.q64.p);
  else time_kernels_t<float>(S, reps, out, S.r32.p, S.s32.p, S.y32.p, S.p32.p, S.q32.p);
}

int status_to_rc(int status) {
  if (status == kSweepTimeout) {
    set_last_error("a bounded wait of a sync-free LDLinv sweep gave up; the solve was abandoned");
    return ACG_ERR_TIMEOUT;
  }
  if (status == kBadInput) {
    set_last_error("the right-hand side has a NaN or infinite entry; x is left at zero");
    return ACG_ERR_INVALID;
  }
  return status;
}

// ============================================================================
// Batched solves: up to 64 right-hand sides per launch
// ============================================================================

int kp_index(int kp) { return kp == 8 ? 0 : kp == 16 ? 1 : kp == 32 ? 2 : 3; }
int round_kp(int k) { return k <= 8 ? 8 : k <= 16 ? 16 : k <= 32 ? 32 : 64; }

template <typename F>
void with_cpl(int kp, F&& f) {
  switch (kp) {
    case 8: f(std::integral_constant<int, 1>()); break;
    case 16: f(std::integral_constant<int, 2>()); break;
    case 32: f(std::integral_constant<int, 4>()); break;
    default: f(std::integral_constant<int, 8>()); break;
  }
}

template <typename T, int CPL, bool kForward>
void enqueue_bsweep(cudaStream_t s, const SolverImpl& S, const T* aux, T* sfwd, T* out, T* mark, int ntasks = -1) {
  const TypedArrays<T> A = arrays_of<T>(S);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(S.bsweep_blocks[plan_index<T>()][kp_index(CPL * kBatchLanes)]);
  cfg.blockDim = dim3(kSweepThreads);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (ntasks < 0) ntasks = kForward ? S.ntasks_fb : S.ntasks_bb;
  ACG_CUDA(cudaLaunchKernelEx(&cfg, kb_sweep<T, CPL, kForward>, ntasks,
                              (const SweepTask*)(kForward ? S.tasks_fb.p : S.tasks_bb.p), kForward ? A.fi : A.bi,
                              kForward ? A.fc : A.bc, aux, (const T*)sfwd, out, mark, S.bsh, S.spin_limit));
}

// Batched forward (s from r) and backward (y from s) sweeps, dense tail included.
// The forward sweep marks y pending and the backward sweep marks s pending
// (head rows; nothing waits on the dense tail's rows), so the next iteration
// finds both vectors ready to be swept.
template <typename T, int CPL>
void enqueue_bforward(cudaStream_t s, const SolverImpl& S, const T* r, T* sv, T* y) {
  enqueue_bsweep<T, CPL, true>(s, S, r, (T*)nullptr, sv, y);
  if (S.dt_K) enqueue_dense<T, CPL>(s, S, true, sv, (T*)nullptr, reinterpret_cast<T*>(S.dt_part.p), &S.bsh->all_done);
}
template <typename T, int CPL>
void enqueue_bbackward(cudaStream_t s, const SolverImpl& S, T* sv, T* y) {
  if (S.dt_K) enqueue_dense<T, CPL>(s, S, false, sv, y, reinterpret_cast<T*>(S.dt_part.p), &S.bsh->all_done);
  enqueue_bsweep<T, CPL, false>(s, S, arrays_of<T>(S).g, sv, y, sv);
}
template <typename T, int CPL>
void enqueue_bsweeps(cudaStream_t s, const SolverImpl& S, const T* r, T* sv, T* y) {
  enqueue_bforward<T, CPL>(s, S, r, sv, y);
  enqueue_bbackward<T, CPL>(s, S, sv, y);
}

template <typename T, int CPL>
void enqueue_biteration(cudaStream_t s, const SolverImpl& S, T* r, T* sv, T* y, T* p, T* q, T* x3, double eps,
                        LoopCtl ctl) {
  constexpr int kp = CPL * kBatchLanes;
  const TypedArrays<T> A = arrays_of<T>(S);
  const int n = S.n;
  kb_spmv<T, CPL, true><<<S.bspmv_blocks[plan_index<T>()][kp_index(kp)], kVecThreads, 0, s>>>(
      n, A.lp, A.li, A.lv, p, q, S.bsh, S.bst, S.bpartials.p);
  const int* vg = S.bvec_blocks[plan_index<T>()];
  kb_pq<T><<<vg[0], kVecThreads, 0, s>>>(n, kp, p, q, S.bst, S.bsh, S.bpartials.p, eps, ctl);
  kb_update<T><<<vg[1], kVecThreads, 0, s>>>(n, kp, x3, p, q, r, S.bst, S.bsh, S.bpartials.p, ctl);
  enqueue_bsweeps<T, CPL>(s, S, r, sv, y);
  kb_yzr<T><<<vg[2], kVecThreads, 0, s>>>(n, kp, y, r, S.bst, S.bsh, S.bpartials.p, eps, ctl);
  kb_pupdate_z<T><<<vg[3], kVecThreads, 0, s>>>(n, kp, y, p, S.bst, S.bsh, S.bpartials.p, eps, ctl);
}

template <int CPL>
cudaGraphExec_t build_batch_fp64_graph(SolverImpl& S, int slot) {
  constexpr int kp = CPL * kBatchLanes;
  cudaStream_t s = S.stream;
  const int n = S.n;
  const size_t N = (size_t)n * kp;
  cudaGraph_t top;
  ACG_CUDA(cudaGraphCreate(&top, 0));
  cudaGraphConditionalHandle h;
  ACG_CUDA(cudaGraphConditionalHandleCreate(&h, top, 1u, cudaGraphCondAssignDefault));
  LoopCtl ctl{h, 1};
  double* x3 = S.bx3_64.p;
  begin_into(s, top, {});
  kb_gather_in<<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.iperm.p, S.bb_ext[slot].p, (long long)n, S.bbm.p, S.bst, S.bsh,
                                                  S.bpartials.p);
  kb_center<double><<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.bbm.p, S.br64.p, x3, S.bs64.p, S.by64.p, S.bst,
                                                       S.bsh, S.bpartials.p, ctl);
  enqueue_bsweeps<double, CPL>(s, S, S.br64.p, S.bs64.p, S.by64.p);
  kb_ysum<double><<<kBVecBlocks, kBVecThreads, 0, s>>>(n, kp, S.by64.p, S.bst, S.bsh, S.bpartials.p, ctl);
  kb_zdot<double><<<kBVecBlocks, kBVecThreads, 0, s>>>(n, kp, S.by64.p, S.br64.p, S.bp64.p, S.bst, S.bsh,
                                                     S.bpartials.p, kEps64, 1, ctl);
  std::vector<cudaGraphNode_t> leaves = capture_leaves(s);
  end_into(s);
  cudaGraph_t body;
  cudaGraphNode_t wnode = add_while(top, leaves, h, &body);
  begin_into(s, body, {});
  enqueue_biteration<double, CPL>(s, S, S.br64.p, S.bs64.p, S.by64.p, S.bp64.p, S.bq64.p, x3, kEps64, ctl);
  end_into(s);
  begin_into(s, top, {wnode});
  kb_take_best<double><<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, x3, S.bxf.p, S.bst);
  kb_true_residual<CPL><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.l_ptr.p, S.l_idx.p, S.l_v64.p, S.bxf.p, S.bbm.p,
                                                           nullptr, S.bst, S.bsh, S.bpartials.p);
  kb_scatter_out<<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.iperm.p, S.bxf.p, S.bx_ext[slot].p, (long long)n, S.bsh);
  end_into(s);
  (void)N;
  cudaGraphExec_t exec;
  ACG_CUDA(cudaGraphInstantiate(&exec, top, 0));
  cudaGraphDestroy(top);
  return exec;
}

template <int CPL>
cudaGraphExec_t build_batch_mixed_graph(SolverImpl& S, int slot) {
  constexpr int kp = CPL * kBatchLanes;
  cudaStream_t s = S.stream;
  const int n = S.n;
  const double eps32 = 1.1920928955078125e-07;
  cudaGraph_t top;
  ACG_CUDA(cudaGraphCreate(&top, 0));
  cudaGraphConditionalHandle ho;
  ACG_CUDA(cudaGraphConditionalHandleCreate(&ho, top, 1u, cudaGraphCondAssignDefault));
  LoopCtl octl{ho, 1};
  begin_into(s, top, {});
  kb_gather_in<<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.iperm.p, S.bb_ext[slot].p, (long long)n, S.bbm.p, S.bst, S.bsh,
                                                  S.bpartials.p);
  kb_center<double><<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.bbm.p, S.br64.p, S.bxf.p, (double*)nullptr,
                                                       (double*)nullptr, S.bst, S.bsh, S.bpartials.p, octl);
  std::vector<cudaGraphNode_t> leaves = capture_leaves(s);
  end_into(s);
  cudaGraph_t obody;
  cudaGraphNode_t onode = add_while(top, leaves, ho, &obody);
  cudaGraphConditionalHandle hi;
  ACG_CUDA(cudaGraphConditionalHandleCreate(&hi, obody, 1u, cudaGraphCondAssignDefault));
  LoopCtl ictl{hi, 1};
  begin_into(s, obody, {});
  kb_outer_prep<float><<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.br64.p, S.br32.p, S.bx3_32.p, S.bs32.p, S.by32.p,
                                                          S.bst, S.bsh, S.bpartials.p, ictl);
  enqueue_bsweeps<float, CPL>(s, S, S.br32.p, S.bs32.p, S.by32.p);
  kb_ysum<float><<<kBVecBlocks, kBVecThreads, 0, s>>>(n, kp, S.by32.p, S.bst, S.bsh, S.bpartials.p, ictl);
  kb_zdot<float><<<kBVecBlocks, kBVecThreads, 0, s>>>(n, kp, S.by32.p, S.br32.p, S.bp32.p, S.bst, S.bsh, S.bpartials.p,
                                                    eps32, 2, ictl);
  std::vector<cudaGraphNode_t> ol = capture_leaves(s);
  end_into(s);
  cudaGraph_t ibody;
  cudaGraphNode_t inode = add_while(obody, ol, hi, &ibody);
  begin_into(s, ibody, {});
  enqueue_biteration<float, CPL>(s, S, S.br32.p, S.bs32.p, S.by32.p, S.bp32.p, S.bq32.p, S.bx3_32.p, eps32, ictl);
  end_into(s);
  begin_into(s, obody, {inode});
  kb_outer_correct<float><<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.bx3_32.p, S.bxf.p, S.bst);
  kb_true_residual<CPL><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.l_ptr.p, S.l_idx.p, S.l_v64.p, S.bxf.p, S.bbm.p,
                                                           S.br64.p, S.bst, S.bsh, S.bpartials.p);
  kb_outer_decide<<<1, kMaxBatch, 0, s>>>(S.bst, S.bsh, kp, octl);
  end_into(s);
  begin_into(s, top, {onode});
  kb_scatter_out<<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.iperm.p, S.bxf.p, S.bx_ext[slot].p, (long long)n, S.bsh);
  end_into(s);
  cudaGraphExec_t exec;
  ACG_CUDA(cudaGraphInstantiate(&exec, top, 0));
  cudaGraphDestroy(top);
  return exec;
}

template <typename T, int CPL>
int batch_occupancy(int sms, int cap) {
  int a = 0, b = 0;
  ACG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, kb_sweep<T, CPL, true>, kSweepThreads, 0));
  ACG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kb_sweep<T, CPL, false>, kSweepThreads, 0));
  int m = std::min(a, b);
  if (cap > 0) m = std::min(m, cap);
  return sms * std::max(1, m);
}

template <typename T, int CPL>
int spmv_occupancy(int sms) {
  int a = 0;
  ACG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, kb_spmv<T, CPL, true>, kVecThreads, 0));
  return sms * std::max(1, a);
}

// Grid of a loop-body vector kernel: every block resident at once, so its
// grid-stride walk ends in one wave (a fixed 592-block grid of a kernel with 3
// resident blocks per SM left a second wave of 148 blocks), and at most
// kVecBlocks, the blocks whose partials the reductions hold.
template <class K>
int vec_occupancy(K kernel, int sms) {
  int a = 0;
  ACG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, kernel, kVecThreads, 0));
  return std::min(kVecBlocks, sms * std::max(1, a));
}

template <typename T>
void vec_grids(int sms, int (&out)[4]) {
  out[0] = vec_occupancy(kb_pq<T>, sms);
  out[1] = vec_occupancy(kb_update<T>, sms);
  out[2] = vec_occupancy(kb_yzr<T>, sms);
  out[3] = vec_occupancy(kb_pupdate_z<T>, sms);
}

// The device-pointer entry points read b where the caller wrote it: order the
// solver's stream after the work already queued on the legacy default stream
// (where a caller without streams of its own writes), without holding up the
// host or any other stream (a device-wide synchronization would stall every
// serving loop and copy on the GPU).  A caller writing b on a stream of its
// own synchronizes that stream first.
void order_after_legacy_stream(SolverImpl& S) {
  if (!S.order_ev) ACG_CUDA(cudaEventCreateWithFlags(&S.order_ev, cudaEventDisableTiming));
  ACG_CUDA(cudaEventRecord(S.order_ev, cudaStreamLegacy));
  ACG_CUDA(cudaStreamWaitEvent(S.stream, S.order_ev, 0));
}

void ensure_batch(SolverImpl& S, int kp) {
  if (!S.bst) {
    ACG_CUDA(cudaMalloc(&S.bst, sizeof(PcgState) * kMaxBatch));
    ACG_CUDA(cudaMalloc(&S.bsh, sizeof(BatchShared)));
    ACG_CUDA(cudaMemset(S.bsh, 0, sizeof(BatchShared)));
    ACG_CUDA(cudaMallocHost(&S.h_bst, sizeof(PcgState) * kMaxBatch));
    S.bpartials.alloc((size_t)4 * (kVecBlocks + kRedGroups) * kMaxBatch);
    int sms = 0;
    ACG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S.device));
    S.bsweep_blocks[0][0] = batch_occupancy<double, 1>(sms, S.batch_bps);
    S.bsweep_blocks[0][1] = batch_occupancy<double, 2>(sms, S.batch_bps);
    S.bsweep_blocks[0][2] = batch_occupancy<double, 4>(sms, S.batch_bps);
    S.bsweep_blocks[0][3] = batch_occupancy<double, 8>(sms, S.batch_bps);
    S.bsweep_blocks[1][0] = batch_occupancy<float, 1>(sms, S.batch_bps);
    S.bsweep_blocks[1][1] = batch_occupancy<float, 2>(sms, S.batch_bps);
    S.bsweep_blocks[1][2] = batch_occupancy<float, 4>(sms, S.batch_bps);
    S.bsweep_blocks[1][3] = batch_occupancy<float, 8>(sms, S.batch_bps);
    vec_grids<double>(sms, S.bvec_blocks[0]);
    vec_grids<float>(sms, S.bvec_blocks[1]);
    S.bspmv_blocks[0][0] = spmv_occupancy<double, 1>(sms);
    S.bspmv_blocks[0][1] = spmv_occupancy<double, 2>(sms);
    S.bspmv_blocks[0][2] = spmv_occupancy<double, 4>(sms);
    S.bspmv_blocks[0][3] = spmv_occupancy<double, 8>(sms);
    S.bspmv_blocks[1][0] = spmv_occupancy<float, 1>(sms);
    S.bspmv_blocks[1][1] = spmv_occupancy<float, 2>(sms);
    S.bspmv_blocks[1][2] = spmv_occupancy<float, 4>(sms);
    S.bspmv_blocks[1][3] = spmv_occupancy<float, 8>(sms);
  }
  if (kp <= S.batch_kp) return;
  // growing the buffers invalidates every captured batch graph
  for (auto& per_slot : S.bexec)
    for (auto& row : per_slot)
      for (auto& e : row)
        if (e) {
          cudaGraphExecDestroy(e);
          e = nullptr;
        }
  const size_t N = (size_t)S.n * kp;
  if (S.async_on) {
    S.bb_ext[1].alloc(N);
    S.bx_ext[1].alloc(N);
  }
  for (DevBuf<double>* b : {&S.bb_ext[0], &S.bx_ext[0], &S.bbm, &S.br64, &S.bxf, &S.bs64, &S.by64, &S.bp64, &S.bq64})
    b->alloc(N);
  S.bx3_64.alloc(3 * N);
  for (DevBuf<float>* b : {&S.br32, &S.bs32, &S.by32, &S.bp32, &S.bq32}) b->alloc(N);
  S.bx3_32.alloc(3 * N);
  S.batch_kp = kp;
}

void init_batch_states(PcgState* h, int kp, double tol, int64_t maxits, double maxtime, int stag_test,
                       double min_inner_tol) {
  std::memset(h, 0, sizeof(PcgState) * kMaxBatch);
  for (int c = 0; c < kp; ++c) {
    h[c].tol = tol;
    h[c].maxtime_s = maxtime;
    h[c].maxits = maxits;
    h[c].stag_test = stag_test;
    h[c].tol_user = tol;
    h[c].maxits_user = maxits;
    h[c].min_inner_tol = min_inner_tol;
    h[c].max_outer = 40;
    h[c].inner_tol = std::min(0.25, std::max(h[c].min_inner_tol, 0.5 * tol));
  }
}

// Per-column results of a batched solve; returns the worst column's code.
int batch_results(int levels, const PcgState* h, int k, int precision, float ms, acg_solve_info* info) {
  int worst = 0;
  for (int c = 0; c < k; ++c) {
    if (info) {
      info[c].iterations = precision == 0 ? h[c].itcnt : h[c].total_its;
      info[c].refinements = precision == 0 ? 0 : h[c].outer_its;
      info[c].relres = h[c].nr;
      info[c].best_relres = precision == 0 ? h[c].bestnr : h[c].nr_true;
      info[c].true_relres = h[c].nr_true;
      info[c].solve_ms = ms;
      info[c].status = h[c].status;
      info[c].levels = levels;
    }
    const int rc = status_to_rc(h[c].status);
    if (rc < 0) return rc;
    worst = std::max(worst, rc);
  }
  return worst;
}

cudaGraphExec_t& batch_graph(SolverImpl& S, int slot, int precision, int kp) {
  cudaGraphExec_t& ge = S.bexec[slot][precision][kp_index(kp)];
  if (!ge) {
    with_cpl(kp, [&](auto cpl) {
      constexpr int C = decltype(cpl)::value;
      ge = precision == 0 ? build_batch_fp64_graph<C>(S, slot) : build_batch_mixed_graph<C>(S, slot);
    });
  }
  return ge;
}

void drain_async(SolverImpl& S);

// Solve k <= 64 right-hand sides (column-major, leading dimensions ldb/ldx)
// in one batched graph launch.
int solve_batch(SolverImpl& S, const double* B, int64_t ldb, double* X, int64_t ldx, int k, cudaMemcpyKind kin,
                cudaMemcpyKind kout, double tol, int64_t maxits, double maxtime, int stag_test, int precision,
                acg_solve_info* info) {
  cudaStream_t s = S.stream;
  const int kp = round_kp(k);
  drain_async(S);  // the asynchronous slots share the batch buffers
  std::unique_lock<std::recursive_mutex> glk(g_device_mu);
  ensure_batch(S, std::max(kp, S.batch_kp));
  cudaGraphExec_t ge = batch_graph(S, 0, precision, kp);
  glk.unlock();
  PcgState* h = S.h_bst;
  init_batch_states(h, kp, tol, maxits, maxtime, stag_test, S.min_inner_tol);
  BatchShared hb = {};
  hb.k = k;
  ACG_CUDA(cudaMemcpyAsync(S.bst, h, sizeof(PcgState) * kp, cudaMemcpyHostToDevice, s));
  ACG_CUDA(cudaMemcpyAsync(S.bsh, &hb, sizeof(BatchShared), cudaMemcpyHostToDevice, s));
  ACG_CUDA(cudaMemcpy2DAsync(S.bb_ext[0].p, sizeof(double) * S.n, B, sizeof(double) * ldb, sizeof(double) * S.n, k,
                             kin, s));
  cudaEvent_t e0, e1;
  ACG_CUDA(cudaEventCreate(&e0));
  ACG_CUDA(cudaEventCreate(&e1));
  ACG_CUDA(cudaEventRecord(e0, s));
  ACG_CUDA(cudaGraphLaunch(ge, s));
  ACG_CUDA(cudaEventRecord(e1, s));
  ACG_CUDA(cudaMemcpy2DAsync(X, sizeof(double) * ldx, S.bx_ext[0].p, sizeof(double) * S.n, sizeof(double) * S.n, k,
                             kout, s));
  ACG_CUDA(cudaMemcpyAsync(h, S.bst, sizeof(PcgState) * kp, cudaMemcpyDeviceToHost, s));
  ACG_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return batch_results(S.nlev, h, k, precision, ms, info);
}

// ============================================================================
// Groups: many graphs in one launch (FP64 PCG per graph)
// ============================================================================

GroupArgs group_args(const SolverImpl& S) {
  return GroupArgs{S.chunks.p, S.seg_first.p, S.seg_nchunk.p, S.seg_cnt.p, S.gpartials.p, S.gstates, S.gflags,
                   S.gsh, S.nseg};
}

cudaGraphExec_t build_group_graph(SolverImpl& S) {
  cudaStream_t s = S.stream;
  const int n = S.n;
  const int nb = S.nchunks;
  const GroupArgs g = group_args(S);
  cudaGraph_t top;
  ACG_CUDA(cudaGraphCreate(&top, 0));
  cudaGraphConditionalHandle h;
  ACG_CUDA(cudaGraphConditionalHandleCreate(&h, top, 1u, cudaGraphCondAssignDefault));
  LoopCtl ctl{h, 1};
  const TypedArrays<double> A = arrays_of<double>(S);
  begin_into(s, top, {});
  // tickets of graphs that stopped while blocks of the same launch were still
  // to start are left incomplete by those blocks: clear them every solve
  ACG_CUDA(cudaMemsetAsync(S.seg_cnt.p, 0, sizeof(unsigned int) * 8 * S.nseg, s));
  kg_gather_in<<<nb, kVecThreads, 0, s>>>(S.perm.p, S.b_ext.p, S.bm.p, g);
  kg_center<double><<<nb, kVecThreads, 0, s>>>(S.bm.p, S.r64.p, S.x3_64.p, S.s64.p, S.y64.p, g, ctl, S.vs64, 0);
  enqueue_sweeps<double>(s, S, S.r64.p, S.s64.p, S.y64.p, S.gflags);
  kg_ysum<double><<<nb, kVecThreads, 0, s>>>(S.y64.p, g, ctl, S.vs64);
  kg_zdot<double><<<nb, kVecThreads, 0, s>>>(S.y64.p, S.r64.p, S.p64.p, g, kEps64, 1, ctl, S.vs64);
  std::vector<cudaGraphNode_t> leaves = capture_leaves(s);
  end_into(s);
  cudaGraph_t body;
  cudaGraphNode_t wnode = add_while(top, leaves, h, &body);
  begin_into(s, body, {});
  kg_spmv<double, 8><<<kVecBlocks, kVecThreads, 0, s>>>(n, A.lp, A.li, A.lv, S.p64.p, S.q64.p, S.gflags);
  kg_pq<double><<<nb, kVecThreads, 0, s>>>(S.p64.p, S.q64.p, g, kEps64, ctl);
  kg_update<double><<<nb, kVecThreads, 0, s>>>(n, S.x3_64.p, S.p64.p, S.q64.p, S.r64.p, S.s64.p, S.y64.p, g, ctl,
                                               S.vs64);
  enqueue_sweeps<double>(s, S, S.r64.p, S.s64.p, S.y64.p, S.gflags);
  kg_ysum<double><<<nb, kVecThreads, 0, s>>>(S.y64.p, g, ctl, S.vs64);
  kg_zdot<double><<<nb, kVecThreads, 0, s>>>(S.y64.p, S.r64.p, S.p64.p, g, kEps64, 0, ctl, S.vs64);
  kg_pupdate<double><<<nb, kVecThreads, 0, s>>>(S.y64.p, S.p64.p, g, S.vs64);
  end_into(s);
  begin_into(s, top, {wnode});
  kg_take_best<double><<<nb, kVecThreads, 0, s>>>(n, S.x3_64.p, S.xf.p, g);
  kg_true_residual<<<nb, kVecThreads, 0, s>>>(S.l_ptr.p, S.l_idx.p, S.l_v64.p, S.xf.p, S.bm.p, nullptr, g);
  k_scatter_out<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, S.xf.p, S.x_ext.p);
  end_into(s);
  cudaGraphExec_t exec;
  ACG_CUDA(cudaGraphInstantiate(&exec, top, 0));
  cudaGraphDestroy(top);
  return exec;
}

// Every graph's FP32 PCG inside its own FP64 refinement (the group form of
// build_mixed_graph): an outer WHILE over refinement steps around an inner
// WHILE over PCG iterations; graphs that finish refining sit out the rest.
cudaGraphExec_t build_group_mixed_graph(SolverImpl& S) {
  cudaStream_t s = S.stream;
  const int n = S.n;
  const int nb = S.nchunks;
  const double eps32 = 1.1920928955078125e-07;
  const GroupArgs g = group_args(S);
  const TypedArrays<float> A = arrays_of<float>(S);
  cudaGraph_t top;
  ACG_CUDA(cudaGraphCreate(&top, 0));
  cudaGraphConditionalHandle ho;
  ACG_CUDA(cudaGraphConditionalHandleCreate(&ho, top, 1u, cudaGraphCondAssignDefault));
  LoopCtl octl{ho, 1};
  begin_into(s, top, {});
  ACG_CUDA(cudaMemsetAsync(S.seg_cnt.p, 0, sizeof(unsigned int) * 8 * S.nseg, s));
  kg_gather_in<<<nb, kVecThreads, 0, s>>>(S.perm.p, S.b_ext.p, S.bm.p, g);
  // r64 = bm, x64 (xf) = 0, per-graph |b| and refinement state
  kg_center<double><<<nb, kVecThreads, 0, s>>>(S.bm.p, S.r64.p, S.xf.p, S.s64.p, S.y64.p, g, octl, S.vs64, 1);
  std::vector<cudaGraphNode_t> leaves = capture_leaves(s);
  end_into(s);

  cudaGraph_t obody;
  cudaGraphNode_t onode = add_while(top, leaves, ho, &obody);
  cudaGraphConditionalHandle hi;
  ACG_CUDA(cudaGraphConditionalHandleCreate(&hi, obody, 1u, cudaGraphCondAssignDefault));
  LoopCtl ictl{hi, 1};
  begin_into(s, obody, {});
  kg_outer_begin<<<1, 256, 0, s>>>(g, ictl);
  kg_outer_prep<float><<<nb, kVecThreads, 0, s>>>(S.r64.p, S.r32.p, S.x3_32.p, S.s32.p, S.y32.p, g, ictl, S.vs32);
  enqueue_sweeps<float>(s, S, S.r32.p, S.s32.p, S.y32.p, S.gflags);
  kg_ysum<float><<<nb, kVecThreads, 0, s>>>(S.y32.p, g, ictl, S.vs32);
  kg_zdot<float><<<nb, kVecThreads, 0, s>>>(S.y32.p, S.r32.p, S.p32.p, g, eps32, 2, ictl, S.vs32);
  std::vector<cudaGraphNode_t> ol = capture_leaves(s);
  end_into(s);

  cudaGraph_t ibody;
  cudaGraphNode_t inode = add_while(obody, ol, hi, &ibody);
  begin_into(s, ibody, {});
  kg_spmv<float, 8><<<kVecBlocks, kVecThreads, 0, s>>>(n, A.lp, A.li, A.lv, S.p32.p, S.q32.p, S.gflags);
  kg_pq<float><<<nb, kVecThreads, 0, s>>>(S.p32.p, S.q32.p, g, eps32, ictl);
  kg_update<float><<<nb, kVecThreads, 0, s>>>(n, S.x3_32.p, S.p32.p, S.q32.p, S.r32.p, S.s32.p, S.y32.p, g, ictl,
                                              S.vs32);
  enqueue_sweeps<float>(s, S, S.r32.p, S.s32.p, S.y32.p, S.gflags);
  kg_ysum<float><<<nb, kVecThreads, 0, s>>>(S.y32.p, g, ictl, S.vs32);
  kg_zdot<float><<<nb, kVecThreads, 0, s>>>(S.y32.p, S.r32.p, S.p32.p, g, eps32, 0, ictl, S.vs32);
  kg_pupdate<float><<<nb, kVecThreads, 0, s>>>(S.y32.p, S.p32.p, g, S.vs32);
  end_into(s);

  begin_into(s, obody, {inode});
  kg_outer_correct<float><<<nb, kVecThreads, 0, s>>>(n, S.x3_32.p, S.xf.p, g);
  kg_true_residual<<<nb, kVecThreads, 0, s>>>(S.l_ptr.p, S.l_idx.p, S.l_v64.p, S.xf.p, S.bm.p, S.r64.p, g);
  kg_outer_decide<<<1, 256, 0, s>>>(g, octl);
  end_into(s);

  begin_into(s, top, {onode});
  k_scatter_out<<<kVecBlocks, kVecThreads, 0, s>>>(n, S.perm.p, S.xf.p, S.x_ext.p);
  end_into(s);
  cudaGraphExec_t exec;
  ACG_CUDA(cudaGraphInstantiate(&exec, top, 0));
  cudaGraphDestroy(top);
  return exec;
}

int solve_group(SolverImpl& S, const double* b, double* x, cudaMemcpyKind kin, cudaMemcpyKind kout, double tol,
                int64_t maxits, double maxtime, int stag_test, int precision, acg_solve_info* info) {
  cudaStream_t s = S.stream;
  cudaGraphExec_t& exec = precision == 0 ? S.gexec : S.gexec_mixed;
  if (!exec) {
    std::lock_guard<std::recursive_mutex> glk(g_device_mu);
    exec = precision == 0 ? build_group_graph(S) : build_group_mixed_graph(S);
  }
  PcgState* h = S.h_gstates;
  std::memset(h, 0, sizeof(PcgState) * S.nseg);
  for (int g = 0; g < S.nseg; ++g) {
    h[g].tol = tol;
    h[g].maxtime_s = maxtime;
    h[g].maxits = maxits;
    h[g].stag_test = stag_test;
    h[g].nvert = S.seg_off[g + 1] - S.seg_off[g];
    h[g].tol_user = tol;
    h[g].maxits_user = maxits;
    h[g].min_inner_tol = S.min_inner_tol;
    h[g].max_outer = 40;
    h[g].inner_tol = std::min(0.25, std::max(h[g].min_inner_tol, 0.5 * tol));
  }
  ACG_CUDA(cudaMemcpyAsync(S.gstates, h, sizeof(PcgState) * S.nseg, cudaMemcpyHostToDevice, s));
  ACG_CUDA(cudaMemcpyAsync(S.b_ext.p, b, sizeof(double) * S.n, kin, s));
  cudaEvent_t e0, e1;
  ACG_CUDA(cudaEventCreate(&e0));
  ACG_CUDA(cudaEventCreate(&e1));
  ACG_CUDA(cudaEventRecord(e0, s));
  ACG_CUDA(cudaGraphLaunch(exec, s));
  ACG_CUDA(cudaEventRecord(e1, s));
  ACG_CUDA(cudaMemcpyAsync(x, S.x_ext.p, sizeof(double) * S.n, kout, s));
  ACG_CUDA(cudaMemcpyAsync(h, S.gstates, sizeof(PcgState) * S.nseg, cudaMemcpyDeviceToHost, s));
  ACG_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int worst = 0;
  for (int g = 0; g < S.nseg; ++g) {
    if (info) {
      info[g].iterations = precision == 0 ? h[g].itcnt : h[g].total_its;
      info[g].refinements = precision == 0 ? 0 : h[g].outer_its;
      info[g].relres = h[g].nr;
      info[g].best_relres = precision == 0 ? h[g].bestnr : h[g].nr_true;
      info[g].true_relres = h[g].nr_true;
      info[g].solve_ms = ms;
      info[g].status = h[g].status;
      info[g].levels = S.nlev;
    }
    const int rc = status_to_rc(h[g].status);
    if (rc < 0) return rc;
    worst = std::max(worst, rc);
  }
  return worst;
}

int solve_column(SolverImpl& S, const double* b, double* x, cudaMemcpyKind kin, cudaMemcpyKind kout, double tol,
                 int64_t maxits, double maxtime, int stag_test, int precision, acg_solve_info* info) {
  cudaStream_t s = S.stream;
  if (!S.exec[precision]) {
    std::lock_guard<std::recursive_mutex> glk(g_device_mu);
    S.exec[precision] = precision == 0 ? build_fp64_graph(S) : build_mixed_graph(S);
  }
  PcgState& h = *S.h_st;
  std::memset(&h, 0, sizeof(PcgState));
  h.tol = tol;
  h.maxtime_s = maxtime;
  h.maxits = maxits;
  h.stag_test = stag_test;
  h.tol_user = tol;
  h.maxits_user = maxits;
  h.min_inner_tol = S.min_inner_tol;
  h.max_outer = 40;
  double it0 = 0.5 * tol;
  h.inner_tol = std::min(0.25, std::max(h.min_inner_tol, it0));
  ACG_CUDA(cudaMemcpyAsync(S.st, &h, sizeof(PcgState), cudaMemcpyHostToDevice, s));
  ACG_CUDA(cudaMemcpyAsync(S.b_ext.p, b, sizeof(double) * S.n, kin, s));
  cudaEvent_t e0, e1;
  ACG_CUDA(cudaEventCreate(&e0));
  ACG_CUDA(cudaEventCreate(&e1));
  ACG_CUDA(cudaEventRecord(e0, s));
  ACG_CUDA(cudaGraphLaunch(S.exec[precision], s));
  ACG_CUDA(cudaEventRecord(e1, s));
  ACG_CUDA(cudaMemcpyAsync(x, S.x_ext.p, sizeof(double) * S.n, kout, s));
  ACG_CUDA(cudaMemcpyAsync(&h, S.st, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
  ACG_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (info) {
    info->iterations = precision == 0 ? h.itcnt : h.total_its;
    info->refinements = precision == 0 ? 0 : h.outer_its;
    info->relres = h.nr;
    info->best_relres = precision == 0 ? h.bestnr : h.nr_true;
    info->true_relres = h.nr_true;
    info->solve_ms = ms;
    info->status = h.status;
    info->levels = S.nlev;
  }
  return status_to_rc(h.status);
}

// Device time per call of the batched kernels for kp columns (see time_kernels_t).
// Captures `reps` calls of body() in one graph, launches it once to warm up
// and once timed; returns the milliseconds per call.
template <typename F>
double graph_ms(cudaStream_t s, int reps, F&& body) {
  cudaGraph_t g;
  ACG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < reps; ++i) body();
  ACG_CUDA(cudaStreamEndCapture(s, &g));
  cudaGraphExec_t ge;
  ACG_CUDA(cudaGraphInstantiate(&ge, g, 0));
  ACG_CUDA(cudaGraphLaunch(ge, s));
  cudaEvent_t e0, e1;
  ACG_CUDA(cudaEventCreate(&e0));
  ACG_CUDA(cudaEventCreate(&e1));
  ACG_CUDA(cudaEventRecord(e0, s));
  ACG_CUDA(cudaGraphLaunch(ge, s));
  ACG_CUDA(cudaEventRecord(e1, s));
  ACG_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  ACG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGraphExecDestroy(ge);
  cudaGraphDestroy(g);
  return (double)ms / reps;
}

template <typename T, int CPL>
void time_batch_t(SolverImpl& S, int reps, acg_kernel_times* out, T* r, T* sv, T* y, T* p, T* q, T* x3) {
  constexpr int kp = CPL * kBatchLanes;
  cudaStream_t s = S.stream;
  ACG_CUDA(cudaMemsetAsync(S.bsh, 0, sizeof(BatchShared), s));
  ACG_CUDA(cudaMemsetAsync(r, 0, sizeof(T) * (size_t)S.n * kp, s));
  ACG_CUDA(cudaMemsetAsync(p, 0, sizeof(T) * (size_t)S.n * kp, s));
  ACG_CUDA(cudaStreamSynchronize(s));
  const TypedArrays<T> A = arrays_of<T>(S);
  const size_t N = (size_t)S.n * kp;
  auto time_graph = [&](auto&& body) -> double { return graph_ms(s, reps, body); };
  auto fill_s = [&]() { k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>((int)N, sv, (T*)nullptr); };
  auto fill_y = [&]() { k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>((int)N, y, (T*)nullptr); };
  const double t_fill = time_graph(fill_s);
  out->spmv_ms = time_graph([&]() {
    kb_spmv<T, CPL, true><<<S.bspmv_blocks[plan_index<T>()][kp_index(kp)], kVecThreads, 0, s>>>(
        S.n, A.lp, A.li, A.lv, p, q, S.bsh, S.bst, S.bpartials.p);
  });
  out->forward_ms = time_graph([&]() {
    fill_s();
    enqueue_bforward<T, CPL>(s, S, r, sv, y);
  }) - t_fill;
  // A backward sweep marks s pending as it consumes it, so each timed backward
  // starts from a saved copy of the forward output (q is free after the
  // mat-vec timing); the copy is timed apart and subtracted like the fills.
  ACG_CUDA(cudaMemcpyAsync(q, sv, sizeof(T) * N, cudaMemcpyDeviceToDevice, s));
  auto restore_s = [&]() { ACG_CUDA(cudaMemcpyAsync(sv, q, sizeof(T) * N, cudaMemcpyDeviceToDevice, s)); };
  const double t_restore = time_graph(restore_s);
  out->backward_ms = time_graph([&]() {
    restore_s();
    fill_y();
    enqueue_bbackward<T, CPL>(s, S, sv, y);
  }) - t_fill - t_restore;
  out->forward_sweep_ms = time_graph([&]() {
    fill_s();
    enqueue_bsweep<T, CPL, true>(s, S, r, (T*)nullptr, sv, y);
  }) - t_fill;
  // the forward sweeps above marked all of y pending: rewrite the tail's rows
  // once, which the backward sweep alone reads and never marks
  if (S.dt_K)
    enqueue_dense<T, CPL>(s, S, false, sv, y, reinterpret_cast<T*>(S.dt_part.p), &S.bsh->all_done);
  // the backward sweep alone reads the tail rows the dense product wrote in
  // the backward_ms runs above, so only the head is marked pending
  auto fill_yh = [&]() {
    k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>((int)((size_t)(S.dt_K ? S.dt_v0 : S.n) * kp), y, (T*)nullptr);
  };
  const double t_fill_h = time_graph(fill_yh);
  out->backward_sweep_ms = time_graph([&]() {
    restore_s();
    fill_yh();
    enqueue_bsweep<T, CPL, false>(s, S, A.g, sv, y, sv);
  }) - t_fill_h - t_restore;
  restore_s();
  out->dense_ms = S.dt_K ? time_graph([&]() {
    enqueue_dense<T, CPL>(s, S, true, sv, (T*)nullptr, reinterpret_cast<T*>(S.dt_part.p), &S.bsh->all_done);
    enqueue_dense<T, CPL>(s, S, false, sv, y, reinterpret_cast<T*>(S.dt_part.p), &S.bsh->all_done);
  }) : 0.0;
  // the loop body's vector kernels, each from the same running state (reset
  // by kb_timing_state before every call; the reset is timed apart)
  {
    ACG_CUDA(cudaMemsetAsync(y, 0, sizeof(T) * N, s));
    ACG_CUDA(cudaMemsetAsync(q, 0, sizeof(T) * N, s));
    ACG_CUDA(cudaMemsetAsync(x3, 0, sizeof(T) * 3 * N, s));
    const double eps = sizeof(T) == 4 ? 1.1920928955078125e-07 : kEps64;
    const LoopCtl none{0, 0};
    auto reset = [&]() { kb_timing_state<<<1, 64, 0, s>>>(S.bst, S.bsh, kp); };
    // the copies without the loop-condition call (the same passes; a profiler
    // measures these, not the loop's own kernels)
    const int* vg = S.bvec_blocks[plan_index<T>()];
    const double t_reset = time_graph(reset);
    out->pq_ms = time_graph([&]() {
      reset();
      kb_pq<T, false><<<vg[0], kVecThreads, 0, s>>>(S.n, kp, p, q, S.bst, S.bsh, S.bpartials.p, eps, none);
    }) - t_reset;
    out->update_ms = time_graph([&]() {
      reset();
      kb_update<T, false><<<vg[1], kVecThreads, 0, s>>>(S.n, kp, x3, p, q, r, S.bst, S.bsh, S.bpartials.p, none);
    }) - t_reset;
    out->yzr_ms = time_graph([&]() {
      reset();
      kb_yzr<T, false><<<vg[2], kVecThreads, 0, s>>>(S.n, kp, y, r, S.bst, S.bsh, S.bpartials.p, eps, none);
    }) - t_reset;
    out->pupdate_ms = time_graph([&]() {
      reset();
      kb_pupdate_z<T, false><<<vg[3], kVecThreads, 0, s>>>(S.n, kp, y, p, S.bst, S.bsh, S.bpartials.p, eps, none);
    }) - t_reset;
    // set-up and wrap-up of a batched solve (FP64 blocks in both precisions)
    {
      const int kk = kp;
      ACG_CUDA(cudaMemcpyAsync(&S.bsh->k, &kk, sizeof(int), cudaMemcpyHostToDevice, s));
      ACG_CUDA(cudaStreamSynchronize(s));
      out->gather_ms = time_graph([&]() {
        kb_gather_in<<<kVecBlocks, kVecThreads, 0, s>>>(S.n, kp, S.iperm.p, S.bb_ext[0].p, (long long)S.n, S.bbm.p,
                                                        S.bst, S.bsh, S.bpartials.p);
      });
      out->scatter_ms = time_graph([&]() {
        kb_scatter_out<<<kVecBlocks, kVecThreads, 0, s>>>(S.n, kp, S.iperm.p, S.bxf.p, S.bx_ext[0].p,
                                                          (long long)S.n, S.bsh);
      });
      out->true_residual_ms = time_graph([&]() {
        kb_true_residual<CPL><<<kVecBlocks, kVecThreads, 0, s>>>(S.n, S.l_ptr.p, S.l_idx.p, S.l_v64.p, S.bxf.p,
                                                                 S.bbm.p, S.br64.p, S.bst, S.bsh, S.bpartials.p);
      });
    }
    const double vec = (double)S.n * kp * sizeof(T);
    out->pq_bytes = 2.0 * vec;       // p, q read
    out->update_bytes = 6.0 * vec;   // x, p, q, r read; x', r written
    out->yzr_bytes = 2.0 * vec;      // y, r read
    out->pupdate_bytes = 3.0 * vec;  // y, p read; p written
  }
  out->iteration_ms = 0.0;
  const int dense_launches = S.dt_K ? 2 : 0;
  // mat-vec, pq, update, two sweeps, kb_yzr, kb_pupdate_z and the dense products
  out->launches_per_iteration = 7 + 2 * dense_launches;
  out->forward_launches = 1 + dense_launches;
  const double vb = sizeof(T), nv = S.n;
  out->spmv_bytes = 4.0 * (nv + 1) + (double)S.nnz_l * (4.0 + vb) + 2.0 * nv * kp * vb;
  out->forward_sweep_bytes = (double)S.nnz_fsweep * (4.0 + vb) + 32.0 * S.ntasks_fb + 3.0 * nv * kp * vb;
  out->backward_sweep_bytes = (double)S.nnz_bsweep * (4.0 + vb) + 32.0 * S.ntasks_bb + nv * vb + 3.0 * nv * kp * vb;
  const double kk = (double)S.dt_K;
  out->dense_bytes = 2.0 * kk * (kk + 1.0) / 2.0 * vb;
  out->forward_bytes = out->forward_sweep_bytes + out->dense_bytes / 2.0;
  out->backward_bytes = out->backward_sweep_bytes + out->dense_bytes / 2.0;
  BatchShared hb;
  ACG_CUDA(cudaMemcpy(&hb, S.bsh, sizeof(BatchShared), cudaMemcpyDeviceToHost));
  if (hb.sweep_error) throw CudaError("a batched sweep wait gave up while timing");
}

// The batched sweeps cut at given levels: for each levels[i] = L, the forward
// sweep over the tasks of levels 0..L and the backward sweep over the tasks of
// levels >= L (swept head levels only), each timed alone from the same inputs
// as in time_batch_t.  The fills and the restore copy that prepare each run
// are timed apart and subtracted.  How the time grows with L shows where the
// DAG's levels cost most: the wide first levels, the long middle, the narrow
// deep end near the critical path.
template <typename T, int CPL>
void time_levels_t(SolverImpl& S, int reps, int npts, const int* levels, double* fwd_ms, double* bwd_ms,
                   int* fwd_tasks, int* bwd_tasks, T* r, T* sv, T* y, T* saved) {
  constexpr int kp = CPL * kBatchLanes;
  cudaStream_t s = S.stream;
  const size_t N = (size_t)S.n * kp;
  ACG_CUDA(cudaMemsetAsync(S.bsh, 0, sizeof(BatchShared), s));
  ACG_CUDA(cudaMemsetAsync(r, 0, sizeof(T) * N, s));
  auto fill_s = [&]() { k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>((int)N, sv, (T*)nullptr); };
  auto fill_yh = [&]() {
    k_fill_pending<T><<<kVecBlocks, kVecThreads, 0, s>>>((int)((size_t)(S.dt_K ? S.dt_v0 : S.n) * kp), y, (T*)nullptr);
  };
  auto restore_s = [&]() { ACG_CUDA(cudaMemcpyAsync(sv, saved, sizeof(T) * N, cudaMemcpyDeviceToDevice, s)); };
  // one whole forward pass (sweep and dense product) gives the backward runs
  // their input s; the dense backward product writes the tail rows of y once
  fill_s();
  enqueue_bforward<T, CPL>(s, S, r, sv, y);
  ACG_CUDA(cudaMemcpyAsync(saved, sv, sizeof(T) * N, cudaMemcpyDeviceToDevice, s));
  if (S.dt_K)
    enqueue_dense<T, CPL>(s, S, false, sv, y, reinterpret_cast<T*>(S.dt_part.p), &S.bsh->all_done);
  ACG_CUDA(cudaStreamSynchronize(s));
  const double t_fill = graph_ms(s, reps, fill_s);
  const double t_back = graph_ms(s, reps, [&]() {
    restore_s();
    fill_yh();
  });
  const int nl = (int)S.tfb_upto.size();
  if (nl == 0 || (int)S.tbb_from.size() != nl) throw InputError("the solver has no batched sweep tables");
  for (int i = 0; i < npts; ++i) {
    const int L = std::min(std::max(levels[i], 0), nl - 1);
    const int tf = S.tfb_upto[L], tb = S.tbb_from[L];
    fwd_tasks[i] = tf;
    bwd_tasks[i] = tb;
    // differences of two timings: a prefix shorter than the timing noise may
    // come out below zero, reported as 0
    fwd_ms[i] = std::max(0.0, graph_ms(s, reps, [&]() {
                                fill_s();
                                if (tf > 0) enqueue_bsweep<T, CPL, true>(s, S, r, (T*)nullptr, sv, y, tf);
                              }) - t_fill);
    bwd_ms[i] = std::max(0.0, graph_ms(s, reps, [&]() {
                                restore_s();
                                fill_yh();
                                if (tb > 0) enqueue_bsweep<T, CPL, false>(s, S, arrays_of<T>(S).g, sv, y, sv, tb);
                              }) - t_back);
  }
  BatchShared hb;
  ACG_CUDA(cudaMemcpy(&hb, S.bsh, sizeof(BatchShared), cudaMemcpyDeviceToHost));
  if (hb.sweep_error) throw CudaError("a batched sweep wait gave up while timing");
}

void time_levels(SolverImpl& S, int precision, int kp, int reps, int npts, const int* levels, double* fwd_ms,
                 double* bwd_ms, int* fwd_tasks, int* bwd_tasks) {
  drain_async(S);
  ensure_batch(S, std::max(kp, S.batch_kp));
  with_cpl(kp, [&](auto cpl) {
    constexpr int C = decltype(cpl)::value;
    if (precision == 0)
      time_levels_t<double, C>(S, reps, npts, levels, fwd_ms, bwd_ms, fwd_tasks, bwd_tasks, S.br64.p, S.bs64.p,
                               S.by64.p, S.bq64.p);
    else
      time_levels_t<float, C>(S, reps, npts, levels, fwd_ms, bwd_ms, fwd_tasks, bwd_tasks, S.br32.p, S.bs32.p,
                              S.by32.p, S.bq32.p);
  });
}

void time_batch(SolverImpl& S, int precision, int kp, int reps, acg_kernel_times* out) {
  drain_async(S);
  ensure_batch(S, std::max(kp, S.batch_kp));
  with_cpl(kp, [&](auto cpl) {
    constexpr int C = decltype(cpl)::value;
    if (precision == 0)
      time_batch_t<double, C>(S, reps, out, S.br64.p, S.bs64.p, S.by64.p, S.bp64.p, S.bq64.p, S.bx3_64.p);
    else
      time_batch_t<float, C>(S, reps, out, S.br32.p, S.bs32.p, S.by32.p, S.bp32.p, S.bq32.p, S.bx3_32.p);
  });
}

}  // namespace
}  // namespace acg

// ============================================================================
// C ABI
// ============================================================================
struct acg_solver {
  acg::SolverImpl impl;
};

// A batched solve enqueued by acg_solve_async.  Its results (the columns'
// final states, the solve time) are copied here when the request is collected:
// by acg_wait, or earlier when its slot is needed by a later request.
struct acg_request {
  acg_solver* h = nullptr;  // null once the solver was destroyed (the results were collected first)
  int slot = 0, k = 0, kp = 0, precision = 0, levels = 0;
  double* x = nullptr;  // host destination
  int64_t ldx = 0;
  bool pinned_x = false;  // page-locked: copied by d2h_stream, else at collection
  bool collected = false;
  int rc = ACG_OK;        // a failure met while collecting
  float ms = 0.f;
  acg::PcgState st[acg::kMaxBatch];
};

namespace acg {
namespace {

void ensure_async(SolverImpl& S) {
  if (S.async_on) return;
  ACG_CUDA(cudaStreamCreateWithFlags(&S.h2d_stream, cudaStreamNonBlocking));
  ACG_CUDA(cudaStreamCreateWithFlags(&S.d2h_stream, cudaStreamNonBlocking));
  for (SolverImpl::AsyncSlot& a : S.slots) {
    ACG_CUDA(cudaEventCreateWithFlags(&a.h2d, cudaEventDisableTiming));
    ACG_CUDA(cudaEventCreate(&a.start));
    ACG_CUDA(cudaEventCreate(&a.done));
    ACG_CUDA(cudaEventCreateWithFlags(&a.d2h, cudaEventDisableTiming));
    ACG_CUDA(cudaMallocHost(&a.h_init, sizeof(PcgState) * kMaxBatch));
    ACG_CUDA(cudaMallocHost(&a.h_out, sizeof(PcgState) * kMaxBatch));
    ACG_CUDA(cudaMallocHost(&a.h_bsh, sizeof(BatchShared)));
  }
  if (S.batch_kp) {
    const size_t N = (size_t)S.n * S.batch_kp;
    S.bb_ext[1].alloc(N);
    S.bx_ext[1].alloc(N);
  }
  S.async_on = true;
}

// Wait for the slot's request to finish and copy its results into it.
void collect(SolverImpl& S, int slot) {
  SolverImpl::AsyncSlot& a = S.slots[slot];
  acg_request* r = a.owner;
  if (!r) return;
  a.owner = nullptr;
  r->collected = true;
  cudaError_t e = cudaEventSynchronize(a.d2h);
  if (e == cudaSuccess && !r->pinned_x)
    e = cudaMemcpy2D(r->x, sizeof(double) * r->ldx, S.bx_ext[slot].p, sizeof(double) * S.n, sizeof(double) * S.n,
                     r->k, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_last_error(std::string("asynchronous solve: ") + cudaGetErrorString(e));
    r->rc = ACG_ERR_CUDA;
    return;
  }
  std::memcpy(r->st, a.h_out, sizeof(PcgState) * r->kp);
  cudaEventElapsedTime(&r->ms, a.start, a.done);
}

void drain_async(SolverImpl& S) {
  if (!S.async_on) return;
  collect(S, 0);
  collect(S, 1);
}

// Enqueue one batched solve of k <= 64 columns from host memory: the copy in
// on h2d_stream, the graph on the solver's stream, the copy out on
// d2h_stream, chained by events.  A slot is reused only after its previous
// request was collected, so its blocks and pinned states are free.
int submit_async(acg_solver* h, const double* B, double* X, int k, int64_t ld, double tol, int64_t maxits,
                 double maxtime, int stag_test, int precision, acg_request** out) {
  SolverImpl& S = h->impl;
  const int kp = round_kp(k);
  std::unique_lock<std::recursive_mutex> glk(g_device_mu);
  ensure_async(S);
  if (kp > S.batch_kp) drain_async(S);  // growing the blocks frees the ones in flight
  ensure_batch(S, std::max(kp, S.batch_kp));
  const int slot = S.next_slot;
  SolverImpl::AsyncSlot& a = S.slots[slot];
  collect(S, slot);
  cudaGraphExec_t ge = batch_graph(S, slot, precision, kp);
  glk.unlock();
  auto req = std::make_unique<acg_request>();
  req->h = h;
  req->slot = slot;
  req->k = k;
  req->kp = kp;
  req->precision = precision;
  req->levels = S.nlev;
  req->x = X;
  req->ldx = ld;
  cudaPointerAttributes pa;
  if (cudaPointerGetAttributes(&pa, X) == cudaSuccess) req->pinned_x = pa.type == cudaMemoryTypeHost;
  else cudaGetLastError();
  init_batch_states(a.h_init, kp, tol, maxits, maxtime, stag_test, S.min_inner_tol);
  *a.h_bsh = BatchShared{};
  a.h_bsh->k = k;
  const size_t row = sizeof(double) * S.n;
  ACG_CUDA(cudaMemcpy2DAsync(S.bb_ext[slot].p, row, B, sizeof(double) * ld, row, k, cudaMemcpyHostToDevice,
                             S.h2d_stream));
  ACG_CUDA(cudaEventRecord(a.h2d, S.h2d_stream));
  ACG_CUDA(cudaStreamWaitEvent(S.stream, a.h2d, 0));
  ACG_CUDA(cudaMemcpyAsync(S.bst, a.h_init, sizeof(PcgState) * kp, cudaMemcpyHostToDevice, S.stream));
  ACG_CUDA(cudaMemcpyAsync(S.bsh, a.h_bsh, sizeof(BatchShared), cudaMemcpyHostToDevice, S.stream));
  ACG_CUDA(cudaEventRecord(a.start, S.stream));
  ACG_CUDA(cudaGraphLaunch(ge, S.stream));
  ACG_CUDA(cudaMemcpyAsync(a.h_out, S.bst, sizeof(PcgState) * kp, cudaMemcpyDeviceToHost, S.stream));
  ACG_CUDA(cudaEventRecord(a.done, S.stream));
  ACG_CUDA(cudaStreamWaitEvent(S.d2h_stream, a.done, 0));
  if (req->pinned_x)
    ACG_CUDA(cudaMemcpy2DAsync(X, sizeof(double) * ld, S.bx_ext[slot].p, row, row, k, cudaMemcpyDeviceToHost,
                               S.d2h_stream));
  ACG_CUDA(cudaEventRecord(a.d2h, S.d2h_stream));
  S.next_slot = slot ^ 1;
  a.owner = req.get();
  *out = req.release();
  return ACG_OK;
}

// ============================================================================
// Serving loop (acg_serve_*): continuous batching in one device-resident loop
// ============================================================================

// The loop graph: WHILE(any slot busy or a request waiting) { one tick }, see
// acg_serve.cuh.  The iteration kernels get no loop handle: a tick whose
// columns all stopped skips the rest of its iteration, and only ks_admit ends
// the loop.
template <int CPL>
cudaGraphExec_t build_serve_graph(SolverImpl& S, int precision, ServeRing* ring, ServeRequest* reqs,
                                  ServeSlots* sl) {
  constexpr int kp = CPL * kBatchLanes;
  cudaStream_t s = S.stream;
  const int n = S.n;
  const double eps32 = 1.1920928955078125e-07;
  const int mixed = precision == 1;
  cudaGraph_t top;
  ACG_CUDA(cudaGraphCreate(&top, 0));
  cudaGraphConditionalHandle h;
  ACG_CUDA(cudaGraphConditionalHandleCreate(&h, top, 1u, cudaGraphCondAssignDefault));
  const LoopCtl ctl{h, 1};
  const LoopCtl none{0, 0};
  cudaGraph_t body;
  add_while(top, {}, h, &body);
  begin_into(s, body, {});
  ks_admit<<<1, kMaxBatch, 0, s>>>(ring, reqs, sl, S.bst, S.bsh, kp, ctl, S.min_inner_tol);
  ks_gather<<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.perm.p, ring, reqs, sl, S.bbm.p, S.bst, S.bsh, S.bpartials.p);
  if (mixed) {
    ks_center<float><<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.bbm.p, S.br64.p, S.br32.p, S.bx3_32.p, S.bxf.p,
                                                        S.bp32.p, sl, S.bst, S.bsh, S.bpartials.p, 1);
    ks_inner_start<float><<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.br64.p, S.br32.p, S.bx3_32.p, S.bp32.p, sl,
                                                             S.bst, S.bsh, S.bpartials.p);
    ks_park<<<1, kMaxBatch, 0, s>>>(sl, S.bst, kp);
    enqueue_biteration<float, CPL>(s, S, S.br32.p, S.bs32.p, S.by32.p, S.bp32.p, S.bq32.p, S.bx3_32.p, eps32, none);
    ks_after_iteration<<<1, kMaxBatch, 0, s>>>(sl, S.bst, kp, 1);
    ks_outer_correct<float><<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.bx3_32.p, S.bxf.p, sl, S.bst);
    kb_true_residual<CPL><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.l_ptr.p, S.l_idx.p, S.l_v64.p, S.bxf.p, S.bbm.p,
                                                             S.br64.p, S.bst, S.bsh, S.bpartials.p, &sl->any_refine);
    ks_outer_decide<<<1, kMaxBatch, 0, s>>>(sl, S.bst, S.bsh, kp);
  } else {
    ks_center<double><<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.bbm.p, S.br64.p, S.br64.p, S.bx3_64.p, S.bxf.p,
                                                         S.bp64.p, sl, S.bst, S.bsh, S.bpartials.p, 0);
    ks_park<<<1, kMaxBatch, 0, s>>>(sl, S.bst, kp);
    enqueue_biteration<double, CPL>(s, S, S.br64.p, S.bs64.p, S.by64.p, S.bp64.p, S.bq64.p, S.bx3_64.p, kEps64,
                                    none);
    ks_after_iteration<<<1, kMaxBatch, 0, s>>>(sl, S.bst, kp, 0);
    ks_take_best<double><<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.bx3_64.p, S.bxf.p, sl, S.bst);
    kb_true_residual<CPL><<<kVecBlocks, kVecThreads, 0, s>>>(n, S.l_ptr.p, S.l_idx.p, S.l_v64.p, S.bxf.p, S.bbm.p,
                                                             nullptr, S.bst, S.bsh, S.bpartials.p, &sl->any_end);
  }
  ks_scatter<<<kVecBlocks, kVecThreads, 0, s>>>(n, kp, S.perm.p, S.bxf.p, ring, reqs, sl);
  ks_finish<<<1, kMaxBatch, 0, s>>>(ring, reqs, sl, S.bst, kp, mixed);
  end_into(s);
  cudaGraphExec_t exec;
  ACG_CUDA(cudaGraphInstantiate(&exec, top, 0));
  cudaGraphDestroy(top);
  return exec;
}

}  // namespace
}  // namespace acg

// A request of acg_serve_submit: nrhs single-right-hand-side solves.
struct acg_ticket {
  struct acg_server* srv = nullptr;
  int k = 0;
  double* x = nullptr;
  int64_t ldx = 0;
  int remaining = 0;
  int rc = ACG_OK;
  std::vector<acg_solve_info> info;
};

struct acg_server {
  acg_solver* h = nullptr;
  int precision = 0, kp = 0, capacity = 0;
  acg::ServeRing* ring_h = nullptr;
  acg::ServeRing* ring_d = nullptr;
  acg::ServeRequest* reqs_h = nullptr;
  acg::ServeRequest* reqs_d = nullptr;
  acg::ServeSlots* slots = nullptr;
  std::vector<double*> bstage, xstage;            // device staging per ring entry
  std::vector<std::pair<acg_ticket*, int>> owner;  // per ring entry: (ticket, column) in flight
  cudaGraphExec_t exec = nullptr;
  cudaStream_t loop_stream = nullptr, in_stream = nullptr, out_stream = nullptr;
  cudaEvent_t loop_done = nullptr;
  std::thread manager;
  std::mutex mu;
  std::condition_variable cv;
  bool closing = false, launched = false;
  unsigned long long published = 0;
  int err = ACG_OK;
  std::string err_msg;
  int device = 0;
  int outstanding = 0;                  // tickets submitted and not yet waited
  int64_t launches = 0, completed = 0;  // loop launches, right-hand sides finished
};

namespace acg {
namespace {

// Ends the ring entry e's request column: x to the caller, info, entry freed.
// Called by the manager thread with srv->mu held.
void serve_complete(acg_server* srv, int e) {
  acg_ticket* t = srv->owner[e].first;
  const int c = srv->owner[e].second;
  const ServeRequest& r = srv->reqs_h[e];
  const int n = srv->h->impl.n;
  cudaError_t ce = cudaMemcpyAsync(t->x + (size_t)c * t->ldx, srv->xstage[e], sizeof(double) * n,
                                   cudaMemcpyDeviceToHost, srv->out_stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(srv->out_stream);
  acg_solve_info& in = t->info[c];
  in.iterations = r.iterations;
  in.refinements = r.refinements;
  in.relres = r.relres;
  in.best_relres = r.true_relres;
  in.true_relres = r.true_relres;
  in.solve_ms = r.solve_ms;
  in.status = r.status;
  in.levels = srv->h->impl.nlev;
  const int rc = ce == cudaSuccess ? status_to_rc(r.status) : ACG_ERR_CUDA;
  if (ce != cudaSuccess) cudaGetLastError();
  if (rc < 0) t->rc = t->rc < 0 ? t->rc : rc;
  else if (t->rc >= 0) t->rc = std::max(t->rc, rc);
  srv->owner[e] = {nullptr, 0};
  t->remaining -= 1;
  srv->completed += 1;
}

// The server's host thread: hands finished solves back, and launches the loop
// graph whenever requests wait and it is not running.  A request published
// just as the loop decided to end is seen here after the launch completes.
void serve_manager(acg_server* srv) {
  cudaSetDevice(srv->device);
  std::unique_lock<std::mutex> lk(srv->mu);
  while (true) {
    bool progress = false;
    for (int e = 0; e < srv->capacity; ++e)
      if (srv->owner[e].first && *(volatile int*)&srv->reqs_h[e].done) {
        serve_complete(srv, e);
        progress = true;
      }
    if (progress) srv->cv.notify_all();
    if (srv->launched && cudaEventQuery(srv->loop_done) == cudaSuccess) {
      srv->launched = false;
      progress = true;
    }
    const unsigned long long head = *(volatile unsigned long long*)&srv->ring_h->head;
    if (!srv->launched && srv->published > head && srv->err == ACG_OK) {
      *(volatile int*)&srv->ring_h->running = 1;
      cudaError_t ce = cudaGraphLaunch(srv->exec, srv->loop_stream);
      if (ce == cudaSuccess) ce = cudaEventRecord(srv->loop_done, srv->loop_stream);
      if (ce != cudaSuccess) {
        cudaGetLastError();
        srv->err = ACG_ERR_CUDA;
        srv->err_msg = std::string("serving loop launch: ") + cudaGetErrorString(ce);
        srv->cv.notify_all();
      } else {
        srv->launched = true;
        srv->launches += 1;
      }
      continue;
    }
    bool busy = false;
    for (int e = 0; e < srv->capacity && !busy; ++e) busy = srv->owner[e].first != nullptr;
    if (srv->closing && !busy && !srv->launched) break;
    if (srv->launched || busy) {
      // the loop runs: poll the done flags
      lk.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(progress ? 0 : 20));
      lk.lock();
    } else {
      srv->cv.wait(lk);
    }
  }
}

}  // namespace
}  // namespace acg

namespace {

template <class F>
int guarded(const char* where, F&& fn) {
  try {
    return fn();
  } catch (const acg::InputError& e) {
    acg::set_last_error(std::string(where) + ": " + e.what());
    return ACG_ERR_INVALID;
  } catch (const acg::DeviceNoMem& e) {
    acg::set_last_error(std::string(where) + ": " + e.what());
    return ACG_ERR_NOMEM;
  } catch (const std::bad_alloc&) {
    acg::set_last_error(std::string(where) + ": host out of memory");
    return ACG_ERR_NOMEM;
  } catch (const acg::CudaError& e) {
    acg::set_last_error(std::string(where) + ": " + e.what());
    return ACG_ERR_CUDA;
  } catch (const std::exception& e) {
    acg::set_last_error(std::string(where) + ": " + e.what());
    return ACG_ERR_INVALID;
  }
}

int check_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    acg::set_last_error(std::string("no CUDA device: ") + cudaGetErrorString(e));
    return ACG_ERR_NODEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    cudaGetLastError();
    acg::set_last_error("cudaGetDeviceProperties failed");
    return ACG_ERR_NODEVICE;
  }
  if (prop.major != 10) {
    acg::set_last_error("libacgpu is built for sm_100a (B200); device " + std::string(prop.name) + " is sm_" +
                        std::to_string(prop.major) + std::to_string(prop.minor));
    return ACG_ERR_NODEVICE;
  }
  return ACG_OK;
}

}  // namespace

extern "C" {

int acg_device_check(void) { return check_device(); }

int acg_create(int64_t n, const int64_t* a_colptr, const int64_t* a_rowval, const double* a_nzval,
               const int64_t* ldli_col, const int64_t* ldli_colptr, const int64_t* ldli_rowval,
               const double* ldli_fval, const double* ldli_d, int64_t ldli_nnz, int index_base,
               const acg_options* opts, acg_solver** out) {
  if (!out || !a_colptr || !a_rowval || !a_nzval || !ldli_col || !ldli_colptr || !ldli_rowval || !ldli_fval ||
      !ldli_d) {
    acg::set_last_error("acg_create: null argument");
    return ACG_ERR_INVALID;
  }
  *out = nullptr;
  int rc = guarded("acg_create", [&]() {
    acg::validate_inputs(n, a_colptr, a_rowval, a_nzval, ldli_col, n - 1, ldli_colptr, ldli_rowval, ldli_fval,
                         ldli_d, ldli_nnz, index_base, 1, nullptr);
    return ACG_OK;
  });
  if (rc != ACG_OK) return rc;
  rc = check_device();
  if (rc != ACG_OK) return rc;
  return guarded("acg_create", [&]() {
    std::lock_guard<std::recursive_mutex> glk(acg::g_device_mu);
    auto* h = new acg_solver();
    try {
      ACG_CUDA(cudaGetDevice(&h->impl.device));
      ACG_CUDA(cudaStreamCreateWithFlags(&h->impl.stream, cudaStreamNonBlocking));
      acg::build_solver(h->impl, n, a_colptr, a_rowval, a_nzval, ldli_col, n - 1, ldli_colptr, ldli_rowval, ldli_fval,
                        ldli_d, ldli_nnz, index_base, opts);
      // set-up of the allocation-free entry point, with this device current
      h->impl.noalloc_scratch = acg::noalloc_scratch_for_current_device(h->impl.device);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return ACG_OK;
  });
}

void acg_destroy(acg_solver* h) {
  if (!h) return;
  if (h->impl.server) acg_serve_close(h->impl.server);
  std::lock_guard<std::recursive_mutex> glk(acg::g_device_mu);
  {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    acg_request* pending[2] = {h->impl.slots[0].owner, h->impl.slots[1].owner};
    acg::drain_async(h->impl);  // requests not yet waited keep their results
    for (acg_request* r : pending)
      if (r) r->h = nullptr;
  }
  cudaStreamSynchronize(h->impl.stream);
  delete h;
}

int acg_solver_stats(const acg_solver* h, acg_stats* out) {
  if (!h || !out) {
    acg::set_last_error("acg_solver_stats: null argument");
    return ACG_ERR_INVALID;
  }
  const acg::SolverImpl& S = h->impl;
  out->n = S.n;
  out->nnz_lap = S.nnz_l;
  out->nnz_factor = S.nnz_f;
  out->levels = S.nlev;
  int wide = 0, thin = 0;
  for (const auto& st : S.plan[1]) (st.thin ? thin : wide)++;
  out->wide_levels = wide;
  out->thin_runs = thin;
  out->sweep_lanes = acg::kLightLanes;
  size_t bytes = 0;
  auto add = [&](const auto& b) { bytes += b.n * sizeof(*b.p); };
  add(S.perm); add(S.lvl_off_d); add(S.l_ptr); add(S.l_idx); add(S.f_ptr); add(S.f_idx); add(S.b_ptr); add(S.b_idx);
  add(S.l_v64); add(S.f_c64); add(S.b_c64); add(S.g64); add(S.l_v32); add(S.f_c32); add(S.b_c32); add(S.g32);
  add(S.b_ext); add(S.x_ext); add(S.bm); add(S.r64); add(S.s64); add(S.y64); add(S.p64); add(S.q64); add(S.x3_64);
  add(S.xf); add(S.r32); add(S.s32); add(S.y32); add(S.p32); add(S.q32); add(S.x3_32); add(S.partials);
  add(S.tasks_f); add(S.tasks_b);
  add(S.bb_ext[0]); add(S.bx_ext[0]); add(S.bb_ext[1]); add(S.bx_ext[1]); add(S.bbm); add(S.br64); add(S.bxf); add(S.bpartials); add(S.br32); add(S.bs32);
  add(S.by32); add(S.bp32); add(S.bq32); add(S.bx3_32); add(S.bs64); add(S.by64); add(S.bp64); add(S.bq64);
  add(S.bx3_64);
  out->device_bytes = (int64_t)bytes;
  out->batch_capacity = S.batch_kp;
  out->tail_levels = S.tail_nl;
  out->tail_vertices = S.tail_nv;
  out->dense_levels = S.dt_K ? S.nlev - S.dt_L0 : 0;
  out->dense_vertices = S.dt_K;
  out->spmv_lanes = S.vl_spmv;
  return ACG_OK;
}

int acg_solve(acg_solver* h, const double* b, double* x, int64_t nrhs, int64_t ldb, double tol, int64_t maxits,
              double maxtime, int stag_test, int precision, acg_solve_info* info) {
  if (!h || !b || !x || nrhs < 0 || (nrhs > 1 && ldb < h->impl.n) || (precision != 0 && precision != 1) ||
      h->impl.nseg > 1) {
    acg::set_last_error("acg_solve: bad arguments (a group solver takes acg_solve_group)");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_solve", [&]() {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    if (h->impl.serving && nrhs > 1) {
      acg::set_last_error("acg_solve: the solver's batch buffers belong to its serving loop");
      return ACG_ERR_BUSY;
    }
    int worst = ACG_OK;
    if (nrhs == 1)
      return acg::solve_column(h->impl, b, x, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, tol, maxits, maxtime,
                               stag_test, precision, info);
    for (int64_t c0 = 0; c0 < nrhs; c0 += acg::kMaxBatch) {
      const int k = (int)std::min<int64_t>(acg::kMaxBatch, nrhs - c0);
      int rc = acg::solve_batch(h->impl, b + c0 * ldb, ldb, x + c0 * ldb, ldb, k, cudaMemcpyHostToDevice,
                                cudaMemcpyDeviceToHost, tol, maxits, maxtime, stag_test, precision,
                                info ? info + c0 : nullptr);
      if (rc < 0) return rc;
      worst = std::max(worst, rc);
    }
    return worst;
  });
}

int acg_solve_async(acg_solver* h, const double* b, double* x, int64_t nrhs, int64_t ldb, double tol,
                    int64_t maxits, double maxtime, int stag_test, int precision, acg_request** out) {
  if (out) *out = nullptr;
  if (h && h->impl.serving) {
    acg::set_last_error("acg_solve_async: the solver's batch buffers belong to its serving loop");
    return ACG_ERR_BUSY;
  }
  if (!h || !b || !x || !out || nrhs < 1 || nrhs > acg::kMaxBatch || ldb < h->impl.n ||
      (precision != 0 && precision != 1) || h->impl.nseg > 1) {
    acg::set_last_error("acg_solve_async: bad arguments (1 <= nrhs <= 64, ldb >= n, one graph)");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_solve_async", [&]() {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    return acg::submit_async(h, b, x, (int)nrhs, ldb, tol, maxits, maxtime, stag_test, precision, out);
  });
}

int acg_poll(acg_request* r) {
  if (!r) {
    acg::set_last_error("acg_poll: null request");
    return ACG_ERR_INVALID;
  }
  acg_solver* h = r->h;
  if (!h) return 1;
  std::lock_guard<std::mutex> lk(h->impl.mu);
  if (r->collected) return 1;
  const cudaError_t e = cudaEventQuery(h->impl.slots[r->slot].d2h);
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) return 0;
  cudaGetLastError();
  acg::set_last_error(std::string("acg_poll: ") + cudaGetErrorString(e));
  return ACG_ERR_CUDA;
}

int acg_wait(acg_request* r, acg_solve_info* info) {
  if (!r) {
    acg::set_last_error("acg_wait: null request");
    return ACG_ERR_INVALID;
  }
  std::unique_ptr<acg_request> own(r);
  return guarded("acg_wait", [&]() {
    acg_solver* h = r->h;
    if (h) {
      cudaEvent_t ev = nullptr;
      {
        std::lock_guard<std::mutex> lk(h->impl.mu);
        if (!r->collected) ev = h->impl.slots[r->slot].d2h;
      }
      if (ev) cudaEventSynchronize(ev);  // without the lock: other threads may submit meanwhile
      std::lock_guard<std::mutex> lk(h->impl.mu);
      if (!r->collected) acg::collect(h->impl, r->slot);
    }
    if (r->rc != ACG_OK) return r->rc;
    return acg::batch_results(r->levels, r->st, r->k, r->precision, r->ms, info);
  });
}

int acg_create_group(int64_t ngraphs, const int64_t* offsets, int64_t n, const int64_t* a_colptr,
                     const int64_t* a_rowval, const double* a_nzval, const int64_t* ldli_col, int64_t ncol,
                     const int64_t* ldli_colptr, const int64_t* ldli_rowval, const double* ldli_fval,
                     const double* ldli_d, int64_t ldli_nnz, int index_base, const acg_options* opts,
                     acg_solver** out) {
  if (!out || !offsets || !a_colptr || !a_rowval || !a_nzval || !ldli_col || !ldli_colptr || !ldli_rowval ||
      !ldli_fval || !ldli_d || ngraphs < 1 || ncol != n - ngraphs) {
    acg::set_last_error("acg_create_group: bad arguments (the union factor must have n - ngraphs columns)");
    return ACG_ERR_INVALID;
  }
  *out = nullptr;
  int rc = guarded("acg_create_group", [&]() {
    acg::validate_inputs(n, a_colptr, a_rowval, a_nzval, ldli_col, ncol, ldli_colptr, ldli_rowval, ldli_fval, ldli_d,
                         ldli_nnz, index_base, ngraphs, offsets);
    return ACG_OK;
  });
  if (rc != ACG_OK) return rc;
  rc = check_device();
  if (rc != ACG_OK) return rc;
  return guarded("acg_create_group", [&]() {
    std::lock_guard<std::recursive_mutex> glk(acg::g_device_mu);
    auto* h = new acg_solver();
    try {
      ACG_CUDA(cudaGetDevice(&h->impl.device));
      ACG_CUDA(cudaStreamCreateWithFlags(&h->impl.stream, cudaStreamNonBlocking));
      acg::build_solver(h->impl, n, a_colptr, a_rowval, a_nzval, ldli_col, ncol, ldli_colptr, ldli_rowval, ldli_fval,
                        ldli_d, ldli_nnz, index_base, opts, ngraphs, offsets);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return ACG_OK;
  });
}

int acg_solve_group(acg_solver* h, const double* b, double* x, double tol, int64_t maxits, double maxtime,
                    int stag_test, int precision, acg_solve_info* info) {
  if (!h || !b || !x || (precision != 0 && precision != 1)) {
    acg::set_last_error("acg_solve_group: bad arguments (precision 0 or 1)");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_solve_group", [&]() {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    // a group of one graph is an ordinary solver: one column, info[0]
    if (h->impl.nseg < 2)
      return acg::solve_column(h->impl, b, x, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, tol, maxits, maxtime,
                               stag_test, precision, info);
    return acg::solve_group(h->impl, b, x, cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, tol, maxits, maxtime,
                            stag_test, precision, info);
  });
}

int acg_solve_device(acg_solver* h, const double* b_dev, double* x_dev, double tol, int64_t maxits, double maxtime,
                     int stag_test, int precision, acg_solve_info* info) {
  if (!h || !b_dev || !x_dev || (precision != 0 && precision != 1)) {
    acg::set_last_error("acg_solve_device: bad arguments");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_solve_device", [&]() {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    acg::order_after_legacy_stream(h->impl);
    return acg::solve_column(h->impl, b_dev, x_dev, cudaMemcpyDeviceToDevice, cudaMemcpyDeviceToDevice, tol, maxits,
                             maxtime, stag_test, precision, info);
  });
}

int acg_solve_batch_device(acg_solver* h, const double* b_dev, double* x_dev, int64_t nrhs, int64_t ld, double tol,
                           int64_t maxits, double maxtime, int stag_test, int precision, acg_solve_info* info) {
  if (!h || !b_dev || !x_dev || nrhs < 1 || ld < h->impl.n || (precision != 0 && precision != 1)) {
    acg::set_last_error("acg_solve_batch_device: bad arguments");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_solve_batch_device", [&]() {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    if (h->impl.serving) {
      acg::set_last_error("acg_solve_batch_device: the solver's batch buffers belong to its serving loop");
      return ACG_ERR_BUSY;
    }
    acg::order_after_legacy_stream(h->impl);
    int worst = ACG_OK;
    for (int64_t c0 = 0; c0 < nrhs; c0 += acg::kMaxBatch) {
      const int k = (int)std::min<int64_t>(acg::kMaxBatch, nrhs - c0);
      int rc = acg::solve_batch(h->impl, b_dev + c0 * ld, ld, x_dev + c0 * ld, ld, k, cudaMemcpyDeviceToDevice,
                                cudaMemcpyDeviceToDevice, tol, maxits, maxtime, stag_test, precision,
                                info ? info + c0 : nullptr);
      if (rc < 0) return rc;
      worst = std::max(worst, rc);
    }
    return worst;
  });
}

int acg_ldlsolve(acg_solver* h, const double* r, double* y, int precision) {
  if (!h || !r || !y || (precision != 0 && precision != 1)) {
    acg::set_last_error("acg_ldlsolve: bad arguments");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_ldlsolve", [&]() {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    acg::SolverImpl& S = h->impl;
    ACG_CUDA(cudaMemcpyAsync(S.b_ext.p, r, sizeof(double) * S.n, cudaMemcpyHostToDevice, S.stream));
    if (precision == 0) acg::ldlsolve_impl<double>(S, S.r64.p, S.s64.p, S.y64.p);
    else acg::ldlsolve_impl<float>(S, S.r32.p, S.s32.p, S.y32.p);
    ACG_CUDA(cudaStreamSynchronize(S.stream));
    acg::PcgState hs;
    ACG_CUDA(cudaMemcpy(&hs, S.st, sizeof(acg::PcgState), cudaMemcpyDeviceToHost));
    if (hs.sweep_error) {
      acg::set_last_error("acg_ldlsolve: a bounded sweep wait gave up");
      return ACG_ERR_TIMEOUT;
    }
    ACG_CUDA(cudaGetLastError());
    ACG_CUDA(cudaMemcpyAsync(y, S.x_ext.p, sizeof(double) * S.n, cudaMemcpyDeviceToHost, S.stream));
    ACG_CUDA(cudaStreamSynchronize(S.stream));
    return ACG_OK;
  });
}

int acg_lap_mul(acg_solver* h, const double* x, double* y, int precision) {
  if (!h || !x || !y || (precision != 0 && precision != 1)) {
    acg::set_last_error("acg_lap_mul: bad arguments");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_lap_mul", [&]() {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    acg::SolverImpl& S = h->impl;
    ACG_CUDA(cudaMemcpyAsync(S.b_ext.p, x, sizeof(double) * S.n, cudaMemcpyHostToDevice, S.stream));
    if (precision == 0) acg::lapmul_impl<double>(S, S.r64.p);
    else acg::lapmul_impl<float>(S, S.r32.p);
    ACG_CUDA(cudaGetLastError());
    ACG_CUDA(cudaMemcpyAsync(y, S.x_ext.p, sizeof(double) * S.n, cudaMemcpyDeviceToHost, S.stream));
    ACG_CUDA(cudaStreamSynchronize(S.stream));
    return ACG_OK;
  });
}

int acg_ldlsolve_noalloc(acg_solver* h, const double* r_dev, double* y_dev, int precision, void* stream) {
  if (!h || !r_dev || !y_dev || (precision != 0 && precision != 1)) {
    acg::set_last_error("acg_ldlsolve_noalloc: bad arguments");
    return ACG_ERR_INVALID;
  }
  if (h->impl.n > ACG_NOALLOC_MAX_N) {
    acg::set_last_error("acg_ldlsolve_noalloc: the graph has " + std::to_string(h->impl.n) +
                        " vertices; the fixed scratch array holds at most " + std::to_string(ACG_NOALLOC_MAX_N));
    return ACG_ERR_INVALID;
  }
  if (h->impl.nseg > 1) {
    acg::set_last_error("acg_ldlsolve_noalloc: needs a one-graph solver from acg_create, not a group solver");
    return ACG_ERR_INVALID;
  }
  if (!h->impl.noalloc_scratch) {
    acg::set_last_error("acg_ldlsolve_noalloc: scratch address was not resolved at acg_create");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_ldlsolve_noalloc", [&]() {
    acg::SolverImpl& S = h->impl;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The factor, the solver's arrays and the scratch address all live on the
    // solver's device; work enqueued on another device would read them as
    // foreign addresses.  Refuse instead of switching devices behind the caller.
    int cur = -1;
    ACG_CUDA(cudaGetDevice(&cur));
    if (cur != S.device)
      throw acg::InputError("the current device is " + std::to_string(cur) + " but the solver lives on device " +
                            std::to_string(S.device));
    if (s) {
      int sdev = -1;
      ACG_CUDA(cudaStreamGetDevice(s, &sdev));
      if (sdev != S.device)
        throw acg::InputError("the stream belongs to device " + std::to_string(sdev) +
                              " but the solver lives on device " + std::to_string(S.device));
    }
    if (precision == 0) acg::ldlsolve_noalloc_impl<double>(S, s, r_dev, y_dev, S.noalloc_scratch);
    else acg::ldlsolve_noalloc_impl<float>(S, s, r_dev, y_dev, S.noalloc_scratch);
    ACG_CUDA(cudaGetLastError());
    ACG_CUDA(cudaStreamSynchronize(s));
    if (acg::noalloc_sweep_error(S.noalloc_scratch)) {
      acg::set_last_error("acg_ldlsolve_noalloc: a bounded sweep wait gave up");
      return ACG_ERR_TIMEOUT;
    }
    return ACG_OK;
  });
}

int acg_time_kernels_batch(acg_solver* h, int precision, int nrhs, int reps, acg_kernel_times* out) {
  if (!h || !out || reps < 1 || nrhs < 1 || nrhs > acg::kMaxBatch || (precision != 0 && precision != 1)) {
    acg::set_last_error("acg_time_kernels_batch: bad arguments");
    return ACG_ERR_INVALID;
  }
  *out = acg_kernel_times{};
  return guarded("acg_time_kernels_batch", [&]() {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    if (h->impl.serving) {
      acg::set_last_error("acg_time_kernels_batch: the solver's batch buffers belong to its serving loop");
      return ACG_ERR_BUSY;
    }
    std::lock_guard<std::recursive_mutex> glk(acg::g_device_mu);
    acg::time_batch(h->impl, precision, acg::round_kp(nrhs), reps, out);
    return ACG_OK;
  });
}

int acg_time_sweep_levels(acg_solver* h, int precision, int nrhs, int reps, int npts, const int* levels,
                          double* fwd_ms, double* bwd_ms, int* fwd_tasks, int* bwd_tasks) {
  if (!h || reps < 1 || nrhs < 1 || nrhs > acg::kMaxBatch || (precision != 0 && precision != 1) || npts < 0 ||
      (npts > 0 && (!levels || !fwd_ms || !bwd_ms || !fwd_tasks || !bwd_tasks))) {
    acg::set_last_error("acg_time_sweep_levels: bad arguments");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_time_sweep_levels", [&]() {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    if (h->impl.serving) {
      acg::set_last_error("acg_time_sweep_levels: the solver's batch buffers belong to its serving loop");
      return ACG_ERR_BUSY;
    }
    if (h->impl.nseg > 1) {
      acg::set_last_error("acg_time_sweep_levels: a group solver has no batched sweeps");
      return ACG_ERR_INVALID;
    }
    std::lock_guard<std::recursive_mutex> glk(acg::g_device_mu);
    acg::time_levels(h->impl, precision, acg::round_kp(nrhs), reps, npts, levels, fwd_ms, bwd_ms, fwd_tasks,
                     bwd_tasks);
    return ACG_OK;
  });
}

int acg_time_kernels(acg_solver* h, int precision, int reps, acg_kernel_times* out) {
  if (!h || !out || reps < 1 || (precision != 0 && precision != 1)) {
    acg::set_last_error("acg_time_kernels: bad arguments");
    return ACG_ERR_INVALID;
  }
  *out = acg_kernel_times{};
  return guarded("acg_time_kernels", [&]() {
    std::lock_guard<std::mutex> lk(h->impl.mu);
    std::lock_guard<std::recursive_mutex> glk(acg::g_device_mu);
    acg::SolverImpl& S = h->impl;
    acg::time_kernels(S, precision, reps, out);
    return ACG_OK;
  });
}

// ---- serving loop -------------------------------------------------------------

int acg_serve_open(acg_solver* h, int precision, int slots, int queue, acg_server** out) {
  if (out) *out = nullptr;
  if (!h || !out || (precision != 0 && precision != 1) || slots < 1 || slots > acg::kMaxBatch || queue < 0 ||
      h->impl.nseg > 1) {
    acg::set_last_error("acg_serve_open: bad arguments (one-graph solver, precision 0 or 1, 1 <= slots <= 64)");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_serve_open", [&]() {
    acg::SolverImpl& S = h->impl;
    std::lock_guard<std::mutex> lk(S.mu);
    std::lock_guard<std::recursive_mutex> glk(acg::g_device_mu);
    if (S.serving) throw acg::InputError("the solver already has a serving loop");
    ACG_CUDA(cudaSetDevice(S.device));
    acg::drain_async(S);
    auto srv = std::make_unique<acg_server>();
    srv->h = h;
    srv->precision = precision;
    srv->device = S.device;
    srv->kp = acg::round_kp(slots);
    srv->capacity = srv->kp + (queue > 0 ? queue : srv->kp);
    acg::ensure_batch(S, std::max(srv->kp, S.batch_kp));
    const size_t ring_bytes = sizeof(acg::ServeRing);
    const size_t reqs_bytes = sizeof(acg::ServeRequest) * srv->capacity;
    ACG_CUDA(cudaHostAlloc(&srv->ring_h, ring_bytes, cudaHostAllocMapped));
    ACG_CUDA(cudaHostAlloc(&srv->reqs_h, reqs_bytes, cudaHostAllocMapped));
    std::memset(srv->ring_h, 0, ring_bytes);
    std::memset(srv->reqs_h, 0, reqs_bytes);
    srv->ring_h->capacity = srv->capacity;
    ACG_CUDA(cudaHostGetDevicePointer((void**)&srv->ring_d, srv->ring_h, 0));
    ACG_CUDA(cudaHostGetDevicePointer((void**)&srv->reqs_d, srv->reqs_h, 0));
    ACG_CUDA(cudaMalloc(&srv->slots, sizeof(acg::ServeSlots)));
    ACG_CUDA(cudaMemset(srv->slots, 0, sizeof(acg::ServeSlots)));
    srv->bstage.assign(srv->capacity, nullptr);
    srv->xstage.assign(srv->capacity, nullptr);
    srv->owner.assign(srv->capacity, {nullptr, 0});
    for (int e = 0; e < srv->capacity; ++e) {
      if (cudaMalloc(&srv->bstage[e], sizeof(double) * S.n) != cudaSuccess ||
          cudaMalloc(&srv->xstage[e], sizeof(double) * S.n) != cudaSuccess) {
        cudaGetLastError();
        for (int f = 0; f <= e; ++f) {
          if (srv->bstage[f]) cudaFree(srv->bstage[f]);
          if (srv->xstage[f]) cudaFree(srv->xstage[f]);
        }
        cudaFree(srv->slots);
        cudaFreeHost(srv->ring_h);
        cudaFreeHost(srv->reqs_h);
        throw acg::DeviceNoMem("serving staging buffers");
      }
    }
    // every slot free and stopped; the batch flags clear
    std::vector<acg::PcgState> st0(acg::kMaxBatch);
    std::memset(st0.data(), 0, sizeof(acg::PcgState) * acg::kMaxBatch);
    for (auto& x : st0) x.done = 1;
    ACG_CUDA(cudaMemcpy(S.bst, st0.data(), sizeof(acg::PcgState) * acg::kMaxBatch, cudaMemcpyHostToDevice));
    ACG_CUDA(cudaMemset(S.bsh, 0, sizeof(acg::BatchShared)));
    {
      // The loop's sweeps find s marked pending by the previous tick's
      // backward sweep, and y by the forward sweep; before the first tick
      // nothing has marked them, so mark both here.  Without this the first
      // forward sweep took whatever the buffer held (zeros, or a freed
      // solver's values) for ready inputs, and the columns admitted in the
      // first tick began their PCG from a wrong z.  The columns' other vectors
      // start at zero, so free slots carry finite values through the sweeps.
      const size_t N = (size_t)S.n * srv->kp;
      for (acg::DevBuf<double>* b : {&S.bbm, &S.br64, &S.bxf, &S.bp64, &S.bq64})
        ACG_CUDA(cudaMemsetAsync(b->p, 0, sizeof(double) * N, S.stream));
      ACG_CUDA(cudaMemsetAsync(S.bx3_64.p, 0, sizeof(double) * 3 * N, S.stream));
      for (acg::DevBuf<float>* b : {&S.br32, &S.bp32, &S.bq32})
        ACG_CUDA(cudaMemsetAsync(b->p, 0, sizeof(float) * N, S.stream));
      ACG_CUDA(cudaMemsetAsync(S.bx3_32.p, 0, sizeof(float) * 3 * N, S.stream));
      acg::k_fill_pending<double><<<acg::kVecBlocks, acg::kVecThreads, 0, S.stream>>>((int)N, S.bs64.p, S.by64.p);
      acg::k_fill_pending<float><<<acg::kVecBlocks, acg::kVecThreads, 0, S.stream>>>((int)N, S.bs32.p, S.by32.p);
      ACG_CUDA(cudaGetLastError());
    }
    acg::with_cpl(srv->kp, [&](auto cpl) {
      constexpr int C = decltype(cpl)::value;
      srv->exec = acg::build_serve_graph<C>(S, precision, srv->ring_d, srv->reqs_d, srv->slots);
    });
    ACG_CUDA(cudaStreamCreateWithFlags(&srv->loop_stream, cudaStreamNonBlocking));
    ACG_CUDA(cudaStreamCreateWithFlags(&srv->in_stream, cudaStreamNonBlocking));
    ACG_CUDA(cudaStreamCreateWithFlags(&srv->out_stream, cudaStreamNonBlocking));
    ACG_CUDA(cudaEventCreateWithFlags(&srv->loop_done, cudaEventDisableTiming));
    ACG_CUDA(cudaStreamSynchronize(S.stream));
    S.serving = true;
    S.server = srv.get();
    acg_server* raw = srv.get();
    raw->manager = std::thread(acg::serve_manager, raw);
    *out = srv.release();
    return ACG_OK;
  });
}

int acg_serve_submit(acg_server* srv, const double* b, double* x, int64_t nrhs, int64_t ldb, double tol,
                     int64_t maxits, double maxtime, int stag_test, acg_ticket** out) {
  if (out) *out = nullptr;
  if (!srv || !b || !x || !out || nrhs < 1 || (nrhs > 1 && ldb < srv->h->impl.n)) {
    acg::set_last_error("acg_serve_submit: bad arguments");
    return ACG_ERR_INVALID;
  }
  return guarded("acg_serve_submit", [&]() {
    const int n = srv->h->impl.n;
    auto t = std::make_unique<acg_ticket>();
    t->srv = srv;
    t->k = (int)nrhs;
    t->x = x;
    t->ldx = nrhs > 1 ? ldb : n;
    t->remaining = (int)nrhs;
    t->info.assign((size_t)nrhs, acg_solve_info{});
    std::unique_lock<std::mutex> lk(srv->mu);
    if (srv->closing) throw acg::InputError("the serving loop is closing");
    for (int64_t c = 0; c < nrhs; ++c) {
      const int e = (int)(srv->published % (unsigned long long)srv->capacity);
      // the entry is reused once its previous request has been completed
      srv->cv.wait(lk, [&]() { return srv->owner[e].first == nullptr || srv->err != ACG_OK; });
      if (srv->err != ACG_OK) throw acg::CudaError(srv->err_msg);
      ACG_CUDA(cudaMemcpyAsync(srv->bstage[e], b + (size_t)c * (nrhs > 1 ? ldb : n), sizeof(double) * n,
                               cudaMemcpyHostToDevice, srv->in_stream));
      ACG_CUDA(cudaStreamSynchronize(srv->in_stream));
      acg::ServeRequest& r = srv->reqs_h[e];
      r.b = srv->bstage[e];
      r.x = srv->xstage[e];
      r.tol = tol;
      r.maxtime = maxtime;
      r.maxits = maxits;
      r.stag_test = stag_test;
      r.done = 0;
      srv->owner[e] = {t.get(), (int)c};
      std::atomic_thread_fence(std::memory_order_seq_cst);
      srv->published += 1;
      *(volatile unsigned long long*)&srv->ring_h->tail = srv->published;
      srv->cv.notify_all();
    }
    srv->outstanding += 1;
    *out = t.release();
    return ACG_OK;
  });
}

int acg_serve_poll(acg_ticket* t) {
  if (!t || !t->srv) {
    acg::set_last_error("acg_serve_poll: null ticket");
    return ACG_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(t->srv->mu);
  if (t->srv->err != ACG_OK) {
    acg::set_last_error(t->srv->err_msg);
    return t->srv->err;
  }
  return t->remaining == 0 ? 1 : 0;
}

int acg_serve_wait(acg_ticket* t, acg_solve_info* info) {
  if (!t || !t->srv) {
    acg::set_last_error("acg_serve_wait: null ticket");
    return ACG_ERR_INVALID;
  }
  std::unique_ptr<acg_ticket> own(t);
  acg_server* srv = t->srv;
  std::unique_lock<std::mutex> lk(srv->mu);
  srv->cv.wait(lk, [&]() { return t->remaining == 0 || srv->err != ACG_OK; });
  srv->outstanding -= 1;
  if (t->remaining != 0) {
    acg::set_last_error(srv->err_msg);
    return srv->err;
  }
  if (info) std::memcpy(info, t->info.data(), sizeof(acg_solve_info) * t->k);
  if (t->rc < 0) acg::set_last_error("acg_serve_wait: a right-hand side failed (see its status)");
  return t->rc;
}

int acg_serve_stats(acg_server* srv, int64_t* launches, int64_t* completed) {
  if (!srv) {
    acg::set_last_error("acg_serve_stats: null server");
    return ACG_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(srv->mu);
  if (launches) *launches = srv->launches;
  if (completed) *completed = srv->completed;
  return ACG_OK;
}

int acg_serve_close(acg_server* srv) {
  if (!srv) return ACG_OK;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->outstanding > 0) {
      acg::set_last_error("acg_serve_close: " + std::to_string(srv->outstanding) + " tickets not yet waited");
      return ACG_ERR_BUSY;
    }
    srv->closing = true;  // requests already published are still served
    srv->cv.notify_all();
  }
  if (srv->manager.joinable()) srv->manager.join();
  acg::SolverImpl& S = srv->h->impl;
  const int rc = srv->err;
  {
    std::lock_guard<std::mutex> lk(S.mu);
    cudaStreamSynchronize(srv->loop_stream);
    if (srv->exec) cudaGraphExecDestroy(srv->exec);
    for (int e = 0; e < srv->capacity; ++e) {
      cudaFree(srv->bstage[e]);
      cudaFree(srv->xstage[e]);
    }
    cudaFree(srv->slots);
    cudaFreeHost(srv->ring_h);
    cudaFreeHost(srv->reqs_h);
    cudaEventDestroy(srv->loop_done);
    cudaStreamDestroy(srv->loop_stream);
    cudaStreamDestroy(srv->in_stream);
    cudaStreamDestroy(srv->out_stream);
    S.serving = false;
    S.server = nullptr;
  }
  delete srv;
  return rc;
}

}  // extern "C"

