// PCG vector kernels with the stop logic of src/pcg.jl:256-445 on the device.
//
// One PCG iteration is the kernel chain
//   k_spmv_pq   q = L p; pq, |p|_1, |q|_1      -> alpha, stagnation tests 1 & 2
//   k_update    x' = x + alpha p; r -= alpha q -> |r|/|b|, bestx, convergence
//   LDLinv sweeps (forward levels, backward levels)  y = LDLinv-apply(r)
//   k_ysum      mean(y)
//   k_zdot      z = y - mean; rho = z.r, |z|_1 -> rho stagnation, inf, beta, test 3,
//                                                 maxtime, maxits
//   k_pupdate   p = z + beta p
// Each reducing kernel finishes its reduction in the last block to arrive
// (grid_reduce) and that block's thread 0 runs the scalar logic.  A finished
// solve sets PcgState::done; every later kernel returns at entry, and the
// graph's loop condition is cleared with cudaGraphSetConditional.
//
// bestx without copies: x lives in three buffers; an update reads
// x[xcur] and writes x[xnext], where xnext is neither the current nor the best
// buffer, so the best iterate is never overwritten.
#pragma once
#include "acg_kernels.cuh"

namespace acg {

enum StopCode {
  kConverged = 0, kMaxits = 1, kStagX = 2, kStagR = 3, kStagRho = 4, kInf = 5, kStagP = 6, kMaxtime = 7,
  kSweepTimeout = 100,  // a bounded device wait of a sweep gave up (reported as an error)
  kBadInput = 101       // the right-hand side has a NaN or infinite entry (reported as an error)
};

struct LoopCtl {
  cudaGraphConditionalHandle handle;
  int use_handle;
};

__device__ __forceinline__ void pcg_stop(PcgState* st, int code, const LoopCtl& ctl) {
  st->status = code;
  st->done = 1;
  if (ctl.use_handle) cudaGraphSetConditional(ctl.handle, 0u);
}

__device__ __forceinline__ int pick_free_buffer(int cur, int best) {
  for (int k = 0; k < 3; ++k)
    if (k != cur && k != best) return k;
  return (cur + 1) % 3;
}

__device__ __forceinline__ bool mark_stop(PcgState* st, int code) {
  st->status = code;
  st->done = 1;
  return true;
}

// ---- scalar steps of one PCG iteration for one system ---------------------
// Each returns true when the system stopped (status and done are then set).
// Shared by the one-right-hand-side kernels (thread 0) and the batched
// kernels (thread c for column c).

// after q = L p: alpha and the first two L1 stagnation tests (src/pcg.jl:288-338)
__device__ __forceinline__ bool pcg_scalar_pq(PcgState* st, double pq, double sum_abs_p, double sum_abs_q,
                                              double eps) {
  if (st->entering) {  // no step yet: x and r stay, the sweeps then give z = pre(r)
    st->alpha = 0.0;
    return false;
  }
  st->itcnt += 1;
  st->sum_abs_p = sum_abs_p;
  st->sum_abs_q = sum_abs_q;
  const double al = st->rho / pq;
  st->alpha = al;
  if (st->itcnt % 10 == 0) {
    if (al * st->sum_abs_p < eps * st->sum_abs_x) return mark_stop(st, kStagX);
    if (al * st->sum_abs_q < eps * st->sum_abs_r) return mark_stop(st, kStagR);
  }
  return false;
}

// after x += alpha p, r -= alpha q: |r|/|b|, bestx, convergence (src/pcg.jl:348-361)
__device__ __forceinline__ bool pcg_scalar_update(PcgState* st, double rr, double sum_abs_x, double sum_abs_r) {
  if (st->entering) return false;
  const double nr = sqrt(rr) / st->nb;
  st->nr = nr;
  st->sum_abs_x = sum_abs_x;
  st->sum_abs_r = sum_abs_r;
  const int xc_new = st->xnext;
  st->xcur = xc_new;
  if (nr < st->bestnr) {
    st->bestnr = nr;
    st->xbest = xc_new;
  }
  st->xnext = pick_free_buffer(xc_new, st->xbest);
  if (nr < st->tol) return mark_stop(st, kConverged);
  return false;
}

// after z = pre(r), rho = z.r: the rho stagnation test, inf and beta
// (src/pcg.jl:365-404).
__device__ __forceinline__ bool pcg_scalar_rho(PcgState* st, double rho) {
  const double oldrho = st->rho;
  st->rho = rho;
  const double thr = 1.0 - 1.0 / (double)st->stag_test;
  if (rho < st->best_rho * thr) {
    st->best_rho = rho;
    st->stag_count = 0;
  } else if (st->stag_test > 0) {
    if (st->best_rho > thr * rho) {
      st->stag_count += 1;
      if (st->stag_count > st->stag_test) return mark_stop(st, kStagRho);
    }
  }
  if (isinf(rho)) return mark_stop(st, kInf);
  const double beta = rho / oldrho;
  st->beta = beta;
  if (isinf(beta)) return mark_stop(st, kInf);
  return false;
}

// the rest of the iteration: the third L1 test (every 10th iteration, with
// st->sum_abs_z of this iteration's z), maxtime and maxits (src/pcg.jl:406-432)
__device__ __forceinline__ bool pcg_scalar_tail(PcgState* st, double eps) {
  if (st->itcnt % 10 == 0 && st->beta * st->sum_abs_p < eps * st->sum_abs_z) return mark_stop(st, kStagP);
  const double el = (double)(globaltimer_ns() - st->t_start) * 1e-9;
  if (el > st->maxtime_s) return mark_stop(st, kMaxtime);
  if (st->itcnt >= st->maxits) return mark_stop(st, kMaxits);
  return false;
}

// The pre-loop step of a system that joined a running serving loop, taken in
// the loop body once its z = pre(r) is known: rho = best_rho = z.r, beta = 0
// (so p = z), as pcg_scalar_zdot's init branch (src/pcg.jl:271-286).
__device__ __forceinline__ bool pcg_scalar_enter(PcgState* st, double zr) {
  st->entering = 0;
  st->rho = zr;
  st->best_rho = zr;
  st->stag_count = 0;
  st->beta = 0.0;
  if (st->itcnt >= st->maxits) return mark_stop(st, kMaxits);
  return false;
}

// after z = pre(r), rho = z.r: stagnation, inf, beta, third L1 test, maxtime,
// maxits (src/pcg.jl:365-432).  init: the pre-loop rho (1 also starts the clock).
__device__ __forceinline__ bool pcg_scalar_zdot(PcgState* st, double zr, double sum_abs_z, double eps, int init) {
  st->sum_abs_z = sum_abs_z;
  if (init) {
    st->rho = zr;
    st->best_rho = zr;
    st->stag_count = 0;
    if (init == 1) st->t_start = globaltimer_ns();
    if (st->itcnt >= st->maxits) return mark_stop(st, kMaxits);
    return false;
  }
  if (pcg_scalar_rho(st, zr)) return true;
  return pcg_scalar_tail(st, eps);
}

__device__ __forceinline__ void clear_loop(const LoopCtl& ctl) {
  if (ctl.use_handle) cudaGraphSetConditional(ctl.handle, 0u);
}

// ---- iteration kernels ---------------------------------------------------

template <typename T, int VL>
__global__ void __launch_bounds__(kVecThreads) k_spmv_pq(int n, const int* __restrict__ ptr, const int* __restrict__ idx,
                                                         const T* __restrict__ val, const T* __restrict__ p, T* __restrict__ q,
                                                         PcgState* st, double* partials, double eps, LoopCtl ctl) {
  if (st->done) return;
  double acc[3] = {0.0, 0.0, 0.0};
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = gt & (VL - 1);
  const int groups = gridDim.x * blockDim.x / VL;
  for (int base = (gt & ~31) / VL; base < n; base += groups) {
    const int row = base + (gt & 31) / VL;
    const bool active = row < n;
    T s = row_dot<T, VL>(ptr, idx, val, p, row, active, lane);
    if (active && lane == 0) {
      q[row] = s;
      const double pr = (double)p[row];
      acc[0] += pr * (double)s;
      acc[1] += fabs(pr);
      acc[2] += fabs((double)s);
    }
  }
  if (grid_reduce<3>(acc, partials, &st->counter[0]) && threadIdx.x == 0)
    if (pcg_scalar_pq(st, acc[0], acc[1], acc[2], eps)) clear_loop(ctl);
}

// Also marks the two sweep output vectors (s, y) pending for the next sweeps.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_update(int n, T* x3, const T* __restrict__ p, const T* __restrict__ q,
                                                        T* __restrict__ r, T* __restrict__ s_out, T* __restrict__ y_out,
                                                        PcgState* st, double* partials, LoopCtl ctl, int vs) {
  if (st->done) return;
  const T pend = pending_value<T>();
  const double al = st->alpha;
  const T* xc = x3 + (size_t)st->xcur * n;
  T* xn = x3 + (size_t)st->xnext * n;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T xv = (T)((double)xc[i] + al * (double)p[i]);
    const T rv = (T)((double)r[i] + (-al) * (double)q[i]);
    xn[i] = xv;
    r[i] = rv;
    s_out[(size_t)i * vs] = pend;
    y_out[(size_t)i * vs] = pend;
    acc[0] += (double)rv * (double)rv;
    acc[1] += fabs((double)xv);
    acc[2] += fabs((double)rv);
  }
  if (grid_reduce<3>(acc, partials, &st->counter[1]) && threadIdx.x == 0)
    if (pcg_scalar_update(st, acc[0], acc[1], acc[2])) clear_loop(ctl);
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_ysum(int n, const T* __restrict__ y, PcgState* st, double* partials,
                                                     LoopCtl ctl, int vs) {
  if (st->done) return;
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[0] += (double)y[(size_t)i * vs];
  if (grid_reduce<1>(acc, partials, &st->counter[2]) && threadIdx.x == 0) {
    st->mean = acc[0] / (double)n;
    if (st->sweep_error) pcg_stop(st, kSweepTimeout, ctl);
  }
}

// z = y - mean (in place); rho = z.r; the rest of the iteration's scalar logic.
// With `init` set this is the pre-loop step: p = z, rho = best_rho = z.r;
// init == 1 (plain PCG) also starts the maxtime clock, init == 2 (an inner
// solve of the refinement loop) keeps the clock started by k_center.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_zdot(int n, T* __restrict__ yz, const T* __restrict__ r, T* __restrict__ p,
                                                      PcgState* st, double* partials, double eps, int init, LoopCtl ctl,
                                                      int vs) {
  if (st->done) return;
  const double mu = st->mean;
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T z = (T)((double)yz[(size_t)i * vs] - mu);
    yz[(size_t)i * vs] = z;
    if (init) p[i] = z;
    acc[0] += (double)z * (double)r[i];
    acc[1] += fabs((double)z);
  }
  if (grid_reduce<2>(acc, partials, &st->counter[3]) && threadIdx.x == 0)
    if (pcg_scalar_zdot(st, acc[0], acc[1], eps, init)) clear_loop(ctl);
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_pupdate(int n, const T* __restrict__ z, T* __restrict__ p, const PcgState* st,
                                                         int vs) {
  if (st->done) return;
  const double beta = st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = (T)((double)z[(size_t)i * vs] + beta * (double)p[i]);
}

// ---- set-up and wrap-up kernels (FP64) ------------------------------------

// b_int[i] = b_ext[perm[i]]; mean(b) -> st->mean.
__global__ void __launch_bounds__(kVecThreads) k_gather_in(int n, const int* __restrict__ perm, const double* __restrict__ bext,
                                                           double* __restrict__ bint, PcgState* st, double* partials) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = bext[perm[i]];
    bint[i] = v;
    acc[0] += v;
  }
  if (grid_reduce<1>(acc, partials, &st->counter[4]) && threadIdx.x == 0) st->mean = acc[0] / (double)n;
}

// bm = b - mean(b); r = bm (cast to T); x buffer 0 = 0; |bm|, |bm|_1; PCG scalars reset.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_center(int n, double* __restrict__ bm, T* __restrict__ r, T* __restrict__ x0,
                                                        T* __restrict__ s_out, T* __restrict__ y_out, PcgState* st,
                                                        double* partials, LoopCtl ctl, int vs) {
  const double mu = st->mean;
  const T pend = pending_value<T>();
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = bm[i] - mu;
    bm[i] = v;
    r[i] = (T)v;
    x0[i] = T(0);
    if (s_out) s_out[(size_t)i * vs] = pend;
    if (y_out) y_out[(size_t)i * vs] = pend;
    acc[0] += v * v;
    acc[1] += fabs(v);
  }
  if (grid_reduce<2>(acc, partials, &st->counter[5]) && threadIdx.x == 0) {
    st->nb = sqrt(acc[0]);
    st->nb64 = st->nb;
    st->scale = st->nb;
    st->sum_abs_r = acc[1];
    st->sum_abs_x = 0.0;
    st->bestnr = 1.0;
    st->nr = 1.0;
    st->nr_true = 1.0;
    st->itcnt = 0;
    st->total_its = 0;
    st->outer_its = 0;
    st->stag_count = 0;
    st->status = kMaxits;
    st->done = 0;
    st->xcur = 0;
    st->xbest = 0;
    st->xnext = 1;
    st->outer_done = 0;
    st->sweep_error = 0;
    st->t_start = globaltimer_ns();
    if (st->nb == 0.0) {
      st->nr_true = 0.0;
      st->nr = 0.0;
      pcg_stop(st, kConverged, ctl);
    } else if (!isfinite(st->nb)) {
      pcg_stop(st, kBadInput, ctl);  // |b| sums every entry: a NaN or Inf shows here
    }
  }
}

// xf = x[xbest] (as double).
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_take_best(int n, const T* __restrict__ x3, double* __restrict__ xf, const PcgState* st) {
  const T* xb = x3 + (size_t)st->xbest * n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) xf[i] = (double)xb[i];
}

// t = bm - L x (FP64); |t|^2 -> relative true residual.  Optionally store t.
template <int VL>
__global__ void __launch_bounds__(kVecThreads) k_true_residual(int n, const int* __restrict__ ptr, const int* __restrict__ idx,
                                                               const double* __restrict__ val, const double* __restrict__ x,
                                                               const double* __restrict__ bm, double* __restrict__ rout,
                                                               PcgState* st, double* partials) {
  double acc[1] = {0.0};
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = gt & (VL - 1);
  const int groups = gridDim.x * blockDim.x / VL;
  for (int base = (gt & ~31) / VL; base < n; base += groups) {
    const int row = base + (gt & 31) / VL;
    const bool active = row < n;
    double s = row_dot<double, VL>(ptr, idx, val, x, row, active, lane);
    if (active && lane == 0) {
      const double t = bm[row] - s;
      if (rout) rout[row] = t;
      acc[0] += t * t;
    }
  }
  if (grid_reduce<1>(acc, partials, &st->counter[6]) && threadIdx.x == 0) {
    st->scale = sqrt(acc[0]);
    st->nr_true = st->nb64 > 0.0 ? st->scale / st->nb64 : 0.0;
  }
}

// x_ext[perm[i]] = xf[i]
__global__ void __launch_bounds__(kVecThreads) k_scatter_out(int n, const int* __restrict__ perm, const double* __restrict__ xf,
                                                             double* __restrict__ xext) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) xext[perm[i]] = xf[i];
}

// ---- mixed precision outer loop ------------------------------------------

// Start of a refinement step: r_in = r64 / scale (FP32); inner PCG state reset.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_outer_prep(int n, const double* __restrict__ r64, T* __restrict__ rin,
                                                            T* __restrict__ x0, T* __restrict__ s_out, T* __restrict__ y_out,
                                                            PcgState* st, double* partials, LoopCtl inner_ctl, int vs) {
  const double inv = 1.0 / st->scale;
  const T pend = pending_value<T>();
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T v = (T)(r64[i] * inv);
    rin[i] = v;
    x0[i] = T(0);
    s_out[(size_t)i * vs] = pend;
    y_out[(size_t)i * vs] = pend;
    acc[0] += (double)v * (double)v;
    acc[1] += fabs((double)v);
  }
  if (grid_reduce<2>(acc, partials, &st->counter[7]) && threadIdx.x == 0) {
    st->nb = sqrt(acc[0]);
    st->sum_abs_r = acc[1];
    st->sum_abs_x = 0.0;
    st->bestnr = 1.0;
    st->nr = 1.0;
    st->itcnt = 0;
    st->stag_count = 0;
    st->status = kMaxits;
    st->done = 0;
    st->xcur = 0;
    st->xbest = 0;
    st->xnext = 1;
    st->tol = st->inner_tol;
    if (inner_ctl.use_handle) cudaGraphSetConditional(inner_ctl.handle, 1u);
    if (st->nb == 0.0) pcg_stop(st, kConverged, inner_ctl);
  }
}

// x64 += scale * x_in[best]
template <typename T>
__global__ void __launch_bounds__(kVecThreads) k_outer_correct(int n, const T* __restrict__ x3, double* __restrict__ x64,
                                                               const PcgState* st) {
  const T* xb = x3 + (size_t)st->xbest * n;
  const double sc = st->scale;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x64[i] += sc * (double)xb[i];
}

// After the true residual: account iterations, decide whether to refine again,
// and give the next inner solve its tolerance and remaining iteration budget.
__global__ void k_outer_decide(PcgState* st, LoopCtl outer_ctl) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  st->total_its += st->itcnt;
  st->outer_its += 1;
  const int inner_status = st->status;
  const bool progressed = st->itcnt > 0 && st->bestnr < 1.0;
  int stop = -1;
  if (st->sweep_error || inner_status == kSweepTimeout) stop = kSweepTimeout;
  else if (st->nr_true <= st->tol_user) stop = kConverged;
  else if (st->total_its >= st->maxits_user) stop = kMaxits;
  else if (st->outer_its >= st->max_outer) stop = kStagX;
  else if (!progressed) stop = inner_status == kMaxits ? kStagRho : inner_status;
  else if ((double)(globaltimer_ns() - st->t_start) * 1e-9 > st->maxtime_s) stop = kMaxtime;
  if (stop >= 0) {
    st->outer_done = 1;
    st->status = stop;
    if (outer_ctl.use_handle) cudaGraphSetConditional(outer_ctl.handle, 0u);
    return;
  }
  double it = 0.5 * st->tol_user / st->nr_true;
  if (it < st->min_inner_tol) it = st->min_inner_tol;
  if (it > 0.25) it = 0.25;
  st->inner_tol = it;
  st->maxits = st->maxits_user - st->total_its;
}

}  // namespace acg
