// Many graphs in one launch: the block-diagonal union of G graphs, each its
// own PCG system with one right-hand side.
//
// Vertices are numbered graph by graph (graph g = internal range
// [seg_off[g], seg_off[g+1])), so every vector of a graph is contiguous; the
// sweeps run the union's task table (level-major across the graphs) in one
// sync-free launch.  The vector kernels run one block per chunk of a graph
// (SegChunk); the last block of a graph to finish sums that graph's block
// partials in block order (deterministic) and runs the scalar PCG step on the
// graph's PcgState.  A graph that stops is counted; when all have stopped the
// loop condition is cleared.  This is the reference's blockSolver
// (src/solverInterface.jl:152-188) with every component solved at once.
#pragma once
#include "acg_pcg.cuh"

namespace acg {

constexpr int kChunk = 2048;  // vector elements per block in the group kernels

struct SegChunk {
  int seg, start, end, pad;
};

struct GroupShared {
  int stopped;         // graphs whose PCG has stopped
  int nseg;
  unsigned int pad[2];
};

struct GroupArgs {
  const SegChunk* chunks;
  const int* seg_first;   // first chunk of each graph
  const int* seg_nchunk;  // chunks of each graph
  unsigned int* seg_cnt;  // [8][nseg] tickets of the per-graph reductions
  double* partials;       // [nchunks][4]
  PcgState* st;           // per graph
  PcgState* gst;          // group flags: done (all stopped), sweep_error
  GroupShared* gsh;
  int nseg;
};

// Block reduction of NV values; the last block of the chunk's graph gets the
// graph totals in tot (thread 0) and returns true.
template <int NV>
__device__ __forceinline__ bool seg_reduce(double (&v)[NV], const SegChunk& c, const GroupArgs& g, int slot,
                                           double (&tot)[NV]) {
  __shared__ double smem[32 * NV];
  __shared__ bool am_last;
  block_reduce<NV>(v, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) g.partials[(size_t)blockIdx.x * 4 + q] = v[q];
    __threadfence();
    unsigned int* cnt = &g.seg_cnt[(size_t)slot * g.nseg + c.seg];
    am_last = atomicAdd(cnt, 1u) == (unsigned int)g.seg_nchunk[c.seg] - 1u;
  }
  __syncthreads();
  if (!am_last) return false;
  if (threadIdx.x == 0) {
    __threadfence();
    const int b0 = g.seg_first[c.seg], nb = g.seg_nchunk[c.seg];
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int b = 0; b < nb; ++b) s += __ldcg(&g.partials[(size_t)(b0 + b) * 4 + q]);
      tot[q] = s;
    }
    g.seg_cnt[(size_t)slot * g.nseg + c.seg] = 0u;
  }
  return true;
}

// A graph stopped: count it; the last one ends the loop.
__device__ __forceinline__ void seg_stopped(const GroupArgs& g, const LoopCtl& ctl) {
  if (atomicAdd(&g.gsh->stopped, 1) + 1 == g.nseg) {
    g.gst->done = 1;
    clear_loop(ctl);
  }
}

template <typename T, int VL>
__global__ void __launch_bounds__(kVecThreads) kg_spmv(int n, const int* __restrict__ ptr, const int* __restrict__ idx,
                                                       const T* __restrict__ val, const T* __restrict__ p,
                                                       T* __restrict__ q, const PcgState* gst) {
  if (gst->done) return;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = gt & (VL - 1);
  const int groups = gridDim.x * blockDim.x / VL;
  for (int base = (gt & ~31) / VL; base < n; base += groups) {
    const int row = base + (gt & 31) / VL;
    const bool active = row < n;
    T s = row_dot<T, VL>(ptr, idx, val, p, row, active, lane);
    if (active && lane == 0) q[row] = s;
  }
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) kg_pq(const T* __restrict__ p, const T* __restrict__ q, GroupArgs g,
                                                     double eps, LoopCtl ctl) {
  if (g.gst->done) return;
  const SegChunk c = g.chunks[blockIdx.x];
  double acc[3] = {0.0, 0.0, 0.0};
  for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) {
    const double pv = (double)p[i], qv = (double)q[i];
    acc[0] += pv * qv;
    acc[1] += fabs(pv);
    acc[2] += fabs(qv);
  }
  double tot[3];
  if (seg_reduce<3>(acc, c, g, 0, tot) && threadIdx.x == 0) {
    PcgState* s = &g.st[c.seg];
    if (!s->done && pcg_scalar_pq(s, tot[0], tot[1], tot[2], eps)) seg_stopped(g, ctl);
  }
}

// x' = x + alpha p, r -= alpha q for graphs still running; s, y pending.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) kg_update(int n, T* x3, const T* __restrict__ p, const T* __restrict__ q,
                                                         T* __restrict__ r, T* __restrict__ s_out, T* __restrict__ y_out,
                                                         GroupArgs g, LoopCtl ctl, int vs) {
  if (g.gst->done) return;
  const SegChunk c = g.chunks[blockIdx.x];
  const PcgState* sc = &g.st[c.seg];
  const bool act = !sc->done;
  const double al = sc->alpha;
  const T* xc = x3 + (size_t)sc->xcur * n;
  T* xn = x3 + (size_t)sc->xnext * n;
  const T pend = pending_value<T>();
  double acc[3] = {0.0, 0.0, 0.0};
  for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) {
    s_out[(size_t)i * vs] = pend;
    y_out[(size_t)i * vs] = pend;
    if (!act) continue;
    const T xv = (T)((double)xc[i] + al * (double)p[i]);
    const T rv = (T)((double)r[i] + (-al) * (double)q[i]);
    xn[i] = xv;
    r[i] = rv;
    acc[0] += (double)rv * (double)rv;
    acc[1] += fabs((double)xv);
    acc[2] += fabs((double)rv);
  }
  double tot[3];
  if (seg_reduce<3>(acc, c, g, 1, tot) && threadIdx.x == 0) {
    PcgState* s = &g.st[c.seg];
    if (!s->done && pcg_scalar_update(s, tot[0], tot[1], tot[2])) seg_stopped(g, ctl);
  }
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) kg_ysum(const T* __restrict__ y, GroupArgs g, LoopCtl ctl, int vs) {
  if (g.gst->done) return;
  const SegChunk c = g.chunks[blockIdx.x];
  double acc[1] = {0.0};
  for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) acc[0] += (double)y[(size_t)i * vs];
  double tot[1];
  if (seg_reduce<1>(acc, c, g, 2, tot) && threadIdx.x == 0) {
    PcgState* s = &g.st[c.seg];
    s->mean = tot[0] / (double)s->nvert;
    if (g.gst->sweep_error && !s->done) {
      mark_stop(s, kSweepTimeout);
      seg_stopped(g, ctl);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) kg_zdot(T* __restrict__ yz, const T* __restrict__ r, T* __restrict__ p,
                                                       GroupArgs g, double eps, int init, LoopCtl ctl, int vs) {
  if (g.gst->done) return;
  const SegChunk c = g.chunks[blockIdx.x];
  const double mu = g.st[c.seg].mean;
  double acc[2] = {0.0, 0.0};
  for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) {
    const T z = (T)((double)yz[(size_t)i * vs] - mu);
    yz[(size_t)i * vs] = z;
    if (init) p[i] = z;
    acc[0] += (double)z * (double)r[i];
    acc[1] += fabs((double)z);
  }
  double tot[2];
  if (seg_reduce<2>(acc, c, g, 3, tot) && threadIdx.x == 0) {
    PcgState* s = &g.st[c.seg];
    if (!s->done && pcg_scalar_zdot(s, tot[0], tot[1], eps, init)) seg_stopped(g, ctl);
  }
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) kg_pupdate(const T* __restrict__ z, T* __restrict__ p, GroupArgs g,
                                                          int vs) {
  if (g.gst->done) return;
  const SegChunk c = g.chunks[blockIdx.x];
  const PcgState* s = &g.st[c.seg];
  if (s->done) return;
  const double beta = s->beta;
  for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x)
    p[i] = (T)((double)z[(size_t)i * vs] + beta * (double)p[i]);
}

// b_int = b_ext[perm]; per-graph sums -> means.  Block 0 also clears the group flags.
__global__ void __launch_bounds__(kVecThreads) kg_gather_in(const int* __restrict__ perm, const double* __restrict__ bext,
                                                            double* __restrict__ bint, GroupArgs g) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    g.gsh->stopped = 0;
    g.gst->done = 0;
    g.gst->sweep_error = 0;
  }
  const SegChunk c = g.chunks[blockIdx.x];
  double acc[1] = {0.0};
  for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) {
    const double v = bext[perm[i]];
    bint[i] = v;
    acc[0] += v;
  }
  double tot[1];
  if (seg_reduce<1>(acc, c, g, 4, tot) && threadIdx.x == 0) g.st[c.seg].mean = tot[0] / (double)g.st[c.seg].nvert;
}

// bm = b - mean; r = bm; x0 = 0; s, y pending; per-graph |b|, state reset.
// outer = 1 starts a mixed-precision solve: the FP64 refinement state is reset
// too, and a graph that stops here is done for the refinement loop as well.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) kg_center(double* __restrict__ bm, T* __restrict__ r, T* __restrict__ x0,
                                                         T* __restrict__ s_out, T* __restrict__ y_out, GroupArgs g,
                                                         LoopCtl ctl, int vs, int outer) {
  const SegChunk c = g.chunks[blockIdx.x];
  const double mu = g.st[c.seg].mean;
  const T pend = pending_value<T>();
  double acc[2] = {0.0, 0.0};
  for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) {
    const double v = bm[i] - mu;
    bm[i] = v;
    r[i] = (T)v;
    x0[i] = T(0);
    s_out[(size_t)i * vs] = pend;
    y_out[(size_t)i * vs] = pend;
    acc[0] += v * v;
    acc[1] += fabs(v);
  }
  double tot[2];
  if (seg_reduce<2>(acc, c, g, 5, tot) && threadIdx.x == 0) {
    PcgState* s = &g.st[c.seg];
    s->nb = sqrt(tot[0]);
    s->nb64 = s->nb;
    s->sum_abs_r = tot[1];
    s->sum_abs_x = 0.0;
    s->bestnr = 1.0;
    s->nr = 1.0;
    s->nr_true = 1.0;
    s->itcnt = 0;
    s->stag_count = 0;
    s->status = kMaxits;
    s->done = 0;
    s->xcur = 0;
    s->xbest = 0;
    s->xnext = 1;
    s->scale = s->nb;
    s->total_its = 0;
    s->outer_its = 0;
    s->outer_done = 0;
    s->t_start = globaltimer_ns();
    if (s->nb == 0.0) {
      s->nr_true = 0.0;
      s->nr = 0.0;
      s->outer_done = outer;
      mark_stop(s, kConverged);
      seg_stopped(g, ctl);
    } else if (!isfinite(s->nb)) {  // a NaN or Inf entry in this graph's right-hand side
      s->outer_done = outer;
      mark_stop(s, kBadInput);
      seg_stopped(g, ctl);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) kg_take_best(int n, const T* __restrict__ x3, double* __restrict__ xf,
                                                            GroupArgs g) {
  const SegChunk c = g.chunks[blockIdx.x];
  const T* xb = x3 + (size_t)g.st[c.seg].xbest * n;
  for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) xf[i] = (double)xb[i];
}

// per graph: t = bm - L xf (FP64), |t| / |bm|.  In a refinement loop (rout
// set) t is stored as the next inner right-hand side, |t| becomes the graph's
// scale, and graphs whose refinement has ended are skipped (every chunk of
// such a graph skips, so its reduction tickets stay balanced).
__global__ void __launch_bounds__(kVecThreads) kg_true_residual(const int* __restrict__ ptr, const int* __restrict__ idx,
                                                                const double* __restrict__ val,
                                                                const double* __restrict__ xf,
                                                                const double* __restrict__ bm,
                                                                double* __restrict__ rout, GroupArgs g) {
  const SegChunk c = g.chunks[blockIdx.x];
  if (rout && g.st[c.seg].outer_done) return;
  double acc[1] = {0.0};
  for (int row = c.start + threadIdx.x; row < c.end; row += blockDim.x) {
    double s = 0.0;
    for (int k = __ldg(&ptr[row]); k < __ldg(&ptr[row + 1]); ++k) s += __ldg(&val[k]) * xf[__ldg(&idx[k])];
    const double t = bm[row] - s;
    if (rout) rout[row] = t;
    acc[0] += t * t;
  }
  double tot[1];
  if (seg_reduce<1>(acc, c, g, 6, tot) && threadIdx.x == 0) {
    PcgState* s = &g.st[c.seg];
    const double nt = sqrt(tot[0]);
    s->nr_true = s->nb64 > 0.0 ? nt / s->nb64 : 0.0;
    if (rout) s->scale = nt;
  }
}

// ---- mixed precision: FP32 PCG inside FP64 refinement, per graph -----------
// The same refinement as one graph's (k_outer_prep .. k_outer_decide): each
// graph keeps its FP64 x and residual, runs FP32 inner PCG on r64 / |r64| to
// an adaptive tolerance, adds |r64| times the inner solution and recomputes
// the true residual; graphs whose refinement has ended sit out the rest.

// Start of a refinement step (one block): the graphs already finished count
// as stopped for the inner loop, which is re-armed.
__global__ void kg_outer_begin(GroupArgs g, LoopCtl inner_ctl) {
  __shared__ int fin;
  if (threadIdx.x == 0) fin = 0;
  __syncthreads();
  int mine = 0;
  for (int q = threadIdx.x; q < g.nseg; q += blockDim.x) mine += g.st[q].outer_done ? 1 : 0;
  atomicAdd(&fin, mine);
  __syncthreads();
  if (threadIdx.x == 0) {
    g.gsh->stopped = fin;
    g.gst->done = fin == g.nseg ? 1 : 0;
    if (inner_ctl.use_handle) cudaGraphSetConditional(inner_ctl.handle, fin == g.nseg ? 0u : 1u);
  }
}

// r_in = r64 / scale (FP32), x buffer 0 = 0, s and y pending; the graph's inner
// PCG state reset (finished graphs are marked done for the inner loop).
template <typename T>
__global__ void __launch_bounds__(kVecThreads) kg_outer_prep(const double* __restrict__ r64, T* __restrict__ rin,
                                                             T* __restrict__ x0, T* __restrict__ s_out,
                                                             T* __restrict__ y_out, GroupArgs g, LoopCtl inner_ctl,
                                                             int vs) {
  const SegChunk c = g.chunks[blockIdx.x];
  PcgState* s = &g.st[c.seg];
  const T pend = pending_value<T>();
  if (s->outer_done) {
    for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) {
      s_out[(size_t)i * vs] = pend;
      y_out[(size_t)i * vs] = pend;
    }
    if (threadIdx.x == 0) s->done = 1;  // every chunk writes the same value
    return;
  }
  const double inv = 1.0 / s->scale;
  double acc[2] = {0.0, 0.0};
  for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) {
    const T v = (T)(r64[i] * inv);
    rin[i] = v;
    x0[i] = T(0);
    s_out[(size_t)i * vs] = pend;
    y_out[(size_t)i * vs] = pend;
    acc[0] += (double)v * (double)v;
    acc[1] += fabs((double)v);
  }
  double tot[2];
  if (seg_reduce<2>(acc, c, g, 7, tot) && threadIdx.x == 0) {
    s->nb = sqrt(tot[0]);
    s->sum_abs_r = tot[1];
    s->sum_abs_x = 0.0;
    s->bestnr = 1.0;
    s->nr = 1.0;
    s->itcnt = 0;
    s->stag_count = 0;
    s->status = kMaxits;
    s->done = 0;
    s->xcur = 0;
    s->xbest = 0;
    s->xnext = 1;
    s->tol = s->inner_tol;
    if (s->nb == 0.0) {
      mark_stop(s, kConverged);
      seg_stopped(g, inner_ctl);
    }
  }
}

// x64 += scale * x_in[best] for the graphs still refining.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) kg_outer_correct(int n, const T* __restrict__ x3,
                                                                double* __restrict__ x64, GroupArgs g) {
  const SegChunk c = g.chunks[blockIdx.x];
  const PcgState* s = &g.st[c.seg];
  if (s->outer_done) return;
  const T* xb = x3 + (size_t)s->xbest * n;
  const double sc = s->scale;
  for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) x64[i] += sc * (double)xb[i];
}

// After the true residuals (one block): per graph, account its iterations and
// decide, as k_outer_decide does for one graph, whether to refine again; the
// refinement loop ends when no graph is left.
__global__ void kg_outer_decide(GroupArgs g, LoopCtl outer_ctl) {
  __shared__ int left;
  if (threadIdx.x == 0) left = 0;
  __syncthreads();
  const bool timeout = g.gst->sweep_error != 0;
  int mine = 0;
  for (int q = threadIdx.x; q < g.nseg; q += blockDim.x) {
    PcgState* st = &g.st[q];
    if (st->outer_done) continue;
    st->total_its += st->itcnt;
    st->outer_its += 1;
    const int inner_status = st->status;
    const bool progressed = st->itcnt > 0 && st->bestnr < 1.0;
    int stop = -1;
    if (timeout || inner_status == kSweepTimeout) stop = kSweepTimeout;
    else if (st->nr_true <= st->tol_user) stop = kConverged;
    else if (st->total_its >= st->maxits_user) stop = kMaxits;
    else if (st->outer_its >= st->max_outer) stop = kStagX;
    else if (!progressed) stop = inner_status == kMaxits ? kStagRho : inner_status;
    else if ((double)(globaltimer_ns() - st->t_start) * 1e-9 > st->maxtime_s) stop = kMaxtime;
    if (stop >= 0) {
      st->outer_done = 1;
      st->status = stop;
      continue;
    }
    double it = 0.5 * st->tol_user / st->nr_true;
    if (it < st->min_inner_tol) it = st->min_inner_tol;
    if (it > 0.25) it = 0.25;
    st->inner_tol = it;
    st->maxits = st->maxits_user - st->total_its;
    ++mine;
  }
  atomicAdd(&left, mine);
  __syncthreads();
  if (threadIdx.x == 0 && left == 0 && outer_ctl.use_handle) cudaGraphSetConditional(outer_ctl.handle, 0u);
}

}  // namespace acg
