// Device-resident serving loop: continuous batching of single-right-hand-side
// solves on one graph.
//
// The batched solver's kp columns are slots.  One CUDA graph launch runs a
// WHILE loop of "ticks"; each tick
//   1. admits requests from a ring in mapped host memory into free slots
//      (ks_admit, one block),
//   2. sets the admitted columns up (ks_gather, ks_center: b - mean(b), |b|,
//      x = 0, p = 0, the column's PCG state) and, in mixed precision, starts
//      the inner FP32 solve of every column that needs one (ks_inner_start),
//   3. runs one PCG iteration of the batched loop body for every running
//      column; a column that has just joined takes its pre-loop step there
//      (PcgState::entering: no update, z = pre(r), rho = z.r, p = z),
//   4. ends the columns that stopped: FP64 takes the best x and its true
//      residual; mixed precision adds the inner solution to its FP64 x,
//      recomputes the true residual and either refines again (next tick) or
//      ends (ks_outer_decide); ended columns' x go to the request's staging
//      buffer and the request is marked done in host memory (ks_finish).
// The loop ends when no slot is busy and the ring is empty; the host relaunches
// it when requests arrive.  Every column is its own PCG system with the
// reference's stop rules (src/pcg.jl:256-445), so a request's result is that
// of the same request solved alone, up to the rounding of its pre-loop rho
// (summed as y.r - mean*(r.1) in the loop body instead of (y - mean).r).
//
// The reference has no server: its closure solves one vector per call
// (src/approxChol.jl:1624).
#pragma once
#include "acg_batch.cuh"

namespace acg {

enum SlotPhase : int {
  kSlotFree = 0,
  kSlotAdmit = 1,      // admitted this tick: set-up pending
  kSlotRun = 2,        // PCG (FP64) or inner FP32 PCG (mixed) running
  kSlotInner = 3,      // mixed: start an inner solve this tick
  kSlotEnd = 4,        // ended this tick: result to the request
};

// One request of the ring (mapped host memory): a single right-hand side.
struct ServeRequest {
  const double* b;     // device staging, n values in the caller's order
  double* x;           // device staging for x
  double tol, maxtime;
  long long maxits;
  int stag_test;
  int pad;
  // written by the device when the solve ends
  long long iterations, refinements;
  double relres, true_relres, solve_ms;
  int status;
  int done;            // set last (after a system-scope fence)
};

struct ServeRing {
  unsigned long long tail;  // requests published by the host
  unsigned long long head;  // requests taken by the device
  int running;              // the device loop is running
  int capacity;
};

// Device-side slot table.
struct ServeSlots {
  int phase[kMaxBatch];
  unsigned long long req[kMaxBatch];  // ring position of each slot's request
  int any_admit, any_inner, any_end, any_refine;
  unsigned long long t_admit[kMaxBatch];
};

// 1. Admission (one block of kMaxBatch threads; thread 0 takes the ring).
__global__ void ks_admit(ServeRing* ring, ServeRequest* reqs, ServeSlots* sl, PcgState* st, BatchShared* bs, int kp,
                         LoopCtl ctl, double min_inner_tol) {
  __shared__ int free_list[kMaxBatch];
  __shared__ int nfree, busy;
  const int c = threadIdx.x;
  if (c == 0) {
    nfree = 0;
    busy = 0;
    sl->any_admit = 0;
    sl->any_inner = 0;
    sl->any_end = 0;
    sl->any_refine = 0;
  }
  __syncthreads();
  if (c < kp) {
    const int ph = sl->phase[c];
    if (ph == kSlotFree) {
      free_list[atomicAdd(&nfree, 1)] = c;
    } else {
      atomicAdd(&busy, 1);
      if (ph == kSlotInner) sl->any_inner = 1;
    }
  }
  __syncthreads();
  if (c == 0) {
    // free slots in increasing order, so that admission is deterministic
    for (int i = 1; i < nfree; ++i)
      for (int j = i; j > 0 && free_list[j - 1] > free_list[j]; --j) {
        const int t = free_list[j];
        free_list[j] = free_list[j - 1];
        free_list[j - 1] = t;
      }
    const unsigned long long tail = *(volatile unsigned long long*)&ring->tail;
    // the host writes an entry before it advances tail: read the entries only
    // after tail (system-scope fence between the loads)
    __threadfence_system();
    unsigned long long head = ring->head;
    int taken = 0;
    while (taken < nfree && head < tail) {
      const int slot = free_list[taken++];
      const volatile ServeRequest& r = reqs[head % (unsigned long long)ring->capacity];
      PcgState* s = &st[slot];
      s->tol = r.tol;
      s->maxtime_s = r.maxtime;
      s->maxits = r.maxits;
      s->stag_test = r.stag_test;
      s->tol_user = r.tol;
      s->maxits_user = r.maxits;
      s->min_inner_tol = min_inner_tol;
      s->max_outer = 40;
      double it = 0.5 * r.tol;
      if (it < s->min_inner_tol) it = s->min_inner_tol;
      if (it > 0.25) it = 0.25;
      s->inner_tol = it;
      sl->req[slot] = head;
      sl->phase[slot] = kSlotAdmit;
      sl->t_admit[slot] = globaltimer_ns();
      ++head;
      sl->any_admit = 1;
    }
    ring->head = head;
    if (busy + taken == 0) {
      // nothing to do: end the loop (the host relaunches it for new requests)
      *(volatile int*)&ring->running = 0;
      __threadfence_system();
      bs->all_done = 1;
      if (ctl.use_handle) cudaGraphSetConditional(ctl.handle, 0u);
    } else {
      bs->all_done = 0;
    }
  }
}

// 2a. Admitted columns: bint[v*kp + c] = b_c[perm[v]], per-column mean.
__global__ void __launch_bounds__(kVecThreads) ks_gather(int n, int kp, const int* __restrict__ perm,
                                                         const ServeRing* ring, const ServeRequest* reqs,
                                                         const ServeSlots* sl, double* __restrict__ bint,
                                                         PcgState* st, BatchShared* bs, double* partials) {
  if (!sl->any_admit) return;
  const size_t N = (size_t)n * kp;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  const bool adm = sl->phase[c] == kSlotAdmit;
  const double* b = adm ? reqs[sl->req[c] % (unsigned long long)ring->capacity].b : nullptr;
  double acc[1] = {0.0};
  if (adm)
    for (size_t i = i0; i < N; i += (size_t)gridDim.x * blockDim.x) {
      const double x = b[perm[i / kp]];
      bint[i] = x;
      acc[0] += x;
    }
  double tot[1];
  if (batch_reduce<1>(acc, kp, partials, &bs->counter[10], tot)) {
    const int cc = threadIdx.x;
    if (cc < kp && sl->phase[cc] == kSlotAdmit) st[cc].mean = tot[0] / (double)n;
  }
}

// 2b. Admitted columns: bm = b - mean; FP64: r = bm, x buffer 0 = 0; mixed:
// x64 = 0 (r64 = bm is the first inner right-hand side); p = 0; |b| and the
// column's state.  A zero right-hand side ends at once (x = 0), a non-finite
// one ends as an input error.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) ks_center(int n, int kp, double* __restrict__ bm, double* __restrict__ r64,
                                                         T* __restrict__ r, T* __restrict__ x0, double* __restrict__ x64,
                                                         T* __restrict__ p, ServeSlots* sl, PcgState* st,
                                                         BatchShared* bs, double* partials, int mixed) {
  if (!sl->any_admit) return;
  const size_t N = (size_t)n * kp;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  const bool adm = sl->phase[c] == kSlotAdmit;
  const double mu = st[c].mean;
  double acc[2] = {0.0, 0.0};
  if (adm)
    for (size_t i = i0; i < N; i += (size_t)gridDim.x * blockDim.x) {
      const double v = bm[i] - mu;
      bm[i] = v;
      if (mixed) {
        r64[i] = v;
        x64[i] = 0.0;
      } else {
        r[i] = (T)v;
        x0[i] = T(0);
      }
      p[i] = T(0);
      acc[0] += v * v;
      acc[1] += fabs(v);
    }
  double tot[2];
  if (batch_reduce<2>(acc, kp, partials, &bs->counter[11], tot)) {
    const int cc = threadIdx.x;
    if (cc < kp && sl->phase[cc] == kSlotAdmit) {
      PcgState* s = &st[cc];
      s->nb = sqrt(tot[0]);
      s->nb64 = s->nb;
      s->scale = s->nb;
      s->sum_abs_r = tot[1];
      s->sum_abs_x = 0.0;
      s->bestnr = 1.0;
      s->nr = 1.0;
      s->nr_true = 1.0;
      s->itcnt = 0;
      s->total_its = 0;
      s->outer_its = 0;
      s->stag_count = 0;
      s->status = kMaxits;
      s->done = 0;
      s->outer_done = 0;
      s->xcur = 0;
      s->xbest = 0;
      s->xnext = 1;
      s->entering = 1;
      s->t_start = globaltimer_ns();
      int ph = mixed ? kSlotInner : kSlotRun;
      if (s->nb == 0.0) {
        s->nr_true = 0.0;
        s->nr = 0.0;
        s->entering = 0;
        mark_stop(s, kConverged);
        ph = kSlotEnd;
      } else if (!isfinite(s->nb)) {
        s->entering = 0;
        mark_stop(s, kBadInput);
        ph = kSlotEnd;
      }
      sl->phase[cc] = ph;
      if (ph == kSlotInner) sl->any_inner = 1;
      if (ph == kSlotEnd) sl->any_end = 1;
    }
  }
}

// 2c. Mixed precision: start the inner FP32 solve of the columns that need one
// (r_in = r64 / scale, x buffer 0 = 0, p = 0, inner state reset, entering).
template <typename T>
__global__ void __launch_bounds__(kVecThreads) ks_inner_start(int n, int kp, const double* __restrict__ r64,
                                                              T* __restrict__ rin, T* __restrict__ x0, T* __restrict__ p,
                                                              ServeSlots* sl, PcgState* st, BatchShared* bs,
                                                              double* partials) {
  if (!sl->any_inner) return;
  const size_t N = (size_t)n * kp;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  const bool go = sl->phase[c] == kSlotInner;
  const double inv = 1.0 / st[c].scale;
  double acc[2] = {0.0, 0.0};
  if (go)
    for (size_t i = i0; i < N; i += (size_t)gridDim.x * blockDim.x) {
      const T v = (T)(r64[i] * inv);
      rin[i] = v;
      x0[i] = T(0);
      p[i] = T(0);
      acc[0] += (double)v * (double)v;
      acc[1] += fabs((double)v);
    }
  double tot[2];
  if (batch_reduce<2>(acc, kp, partials, &bs->counter[12], tot)) {
    const int cc = threadIdx.x;
    if (cc < kp && sl->phase[cc] == kSlotInner) {
      PcgState* s = &st[cc];
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
      s->entering = 1;
      sl->phase[cc] = kSlotRun;
      if (s->nb == 0.0) {
        s->entering = 0;
        mark_stop(s, kConverged);
      }
    }
  }
}

// Free and ended slots take no part in the iteration: mark them stopped.
__global__ void ks_park(ServeSlots* sl, PcgState* st, int kp) {
  const int c = threadIdx.x;
  if (c < kp && sl->phase[c] != kSlotRun) st[c].done = 1;
}

// 4a. After the iteration: a running column that stopped ends (FP64) or
// refines (mixed).
__global__ void ks_after_iteration(ServeSlots* sl, const PcgState* st, int kp, int mixed) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  const int c = threadIdx.x;
  if (c < kp && sl->phase[c] == kSlotRun && st[c].done) {
    sl->phase[c] = kSlotEnd;  // mixed: provisional, ks_outer_decide settles it
    any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0 && any) {
    if (mixed) sl->any_refine = 1;
    else sl->any_end = 1;
  }
}

// 4b. Mixed: x64 += scale * x_in[best] for the columns that finished an inner solve.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) ks_outer_correct(int n, int kp, const T* __restrict__ x3,
                                                                double* __restrict__ x64, const ServeSlots* sl,
                                                                const PcgState* st) {
  if (!sl->any_refine) return;
  const size_t N = (size_t)n * kp;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  if (sl->phase[c] != kSlotEnd) return;
  const T* xb = x3 + (size_t)st[c].xbest * N;
  const double sc = st[c].scale;
  for (size_t i = i0; i < N; i += (size_t)gridDim.x * blockDim.x) x64[i] += sc * (double)xb[i];
}

// 4c. Mixed: per refining column, account the inner iterations and decide as
// k_outer_decide does: end, or start another inner solve next tick.
__global__ void ks_outer_decide(ServeSlots* sl, PcgState* st, BatchShared* bs, int kp) {
  if (!sl->any_refine) return;
  __shared__ int any_end, any_inner;
  if (threadIdx.x == 0) {
    any_end = 0;
    any_inner = 0;
  }
  __syncthreads();
  const int c = threadIdx.x;
  if (c < kp && sl->phase[c] == kSlotEnd) {
    PcgState* s = &st[c];
    s->total_its += s->itcnt;
    s->outer_its += 1;
    const int inner_status = s->status;
    const bool progressed = s->itcnt > 0 && s->bestnr < 1.0;
    int stop = -1;
    if (bs->sweep_error || inner_status == kSweepTimeout) stop = kSweepTimeout;
    else if (s->nr_true <= s->tol_user) stop = kConverged;
    else if (s->total_its >= s->maxits_user) stop = kMaxits;
    else if (s->outer_its >= s->max_outer) stop = kStagX;
    else if (!progressed) stop = inner_status == kMaxits ? kStagRho : inner_status;
    else if ((double)(globaltimer_ns() - s->t_start) * 1e-9 > s->maxtime_s) stop = kMaxtime;
    if (stop >= 0) {
      s->outer_done = 1;
      s->status = stop;
      any_end = 1;
    } else {
      double it = 0.5 * s->tol_user / s->nr_true;
      if (it < s->min_inner_tol) it = s->min_inner_tol;
      if (it > 0.25) it = 0.25;
      s->inner_tol = it;
      s->maxits = s->maxits_user - s->total_its;
      sl->phase[c] = kSlotInner;
      any_inner = 1;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (any_end) sl->any_end = 1;
    if (any_inner) sl->any_inner = 1;
  }
}

// 4d. FP64: the ended columns' best x (as double) into xf.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) ks_take_best(int n, int kp, const T* __restrict__ x3,
                                                            double* __restrict__ xf, const ServeSlots* sl,
                                                            const PcgState* st) {
  if (!sl->any_end) return;
  const size_t N = (size_t)n * kp;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  if (sl->phase[c] != kSlotEnd) return;
  const T* xb = x3 + (size_t)st[c].xbest * N;
  for (size_t i = i0; i < N; i += (size_t)gridDim.x * blockDim.x) xf[i] = (double)xb[i];
}

// 4e. The ended columns' x to their requests' staging buffers (caller's order).
__global__ void __launch_bounds__(kVecThreads) ks_scatter(int n, int kp, const int* __restrict__ perm,
                                                          const double* __restrict__ xf, const ServeRing* ring,
                                                          const ServeRequest* reqs, const ServeSlots* sl) {
  if (!sl->any_end) return;
  const size_t N = (size_t)n * kp;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  if (sl->phase[c] != kSlotEnd) return;
  double* x = reqs[sl->req[c] % (unsigned long long)ring->capacity].x;
  for (size_t i = i0; i < N; i += (size_t)gridDim.x * blockDim.x) x[perm[i / kp]] = xf[i];
}

// 4f. Report the ended requests to the host and free their slots.
__global__ void ks_finish(const ServeRing* ring, ServeRequest* reqs, ServeSlots* sl, const PcgState* st, int kp,
                          int mixed) {
  if (!sl->any_end) return;
  const int c = threadIdx.x;
  const bool end = c < kp && sl->phase[c] == kSlotEnd;
  if (end) {
    ServeRequest& r = reqs[sl->req[c] % (unsigned long long)ring->capacity];
    const PcgState* s = &st[c];
    r.iterations = mixed ? s->total_its : s->itcnt;
    r.refinements = mixed ? s->outer_its : 0;
    r.relres = s->nr;
    r.true_relres = s->nr_true;
    r.solve_ms = (double)(globaltimer_ns() - sl->t_admit[c]) * 1e-6;
    r.status = s->status;
  }
  // the x staging writes of ks_scatter (an earlier kernel) and the fields
  // above reach the host before it sees done
  __threadfence_system();
  __syncthreads();
  if (end) {
    ServeRequest& r = reqs[sl->req[c] % (unsigned long long)ring->capacity];
    *(volatile int*)&r.done = 1;
    sl->phase[c] = kSlotFree;
  }
}

}  // namespace acg
