// Device kernels of the solve phase.
//
// Vertex numbering on the device ("internal" ids) is the forward level order
// of the LDLinv dependency graph: vertices of level 0 first, then level 1,
// ...; inside a level, by elimination step.  Every level is therefore a
// contiguous id range, for both sweeps (the backward sweep walks the same
// levels in reverse).
//
// Factor coefficients.  For the entry e of the column eliminated at vertex u
// (src/approxChol.jl:1369-1408) define
//     coef_e = fval_e * prod_{k<e, k non-last}(1 - fval_k)    (non-last entries)
//     coef_e = P_u   = prod_{k non-last}(1 - fval_k)          (the last entry)
// Then, with s the forward values (y just after forward!):
//     forward   s_j = r_j + sum_{e: row(e)=j} coef_e * s_{col(e)}
//     backward  y_u = g_u * s_u + sum_{e in col(u)} coef_e * y_{row(e)}
// where g_u = P_u * P_u / d_u (g = 1 for the never-eliminated vertex, d = 0).
// This is the reference's forward!/division/backward! with the running
// products folded into per-entry constants (same operator, rounding differs
// in the last bits).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>

namespace acg {

constexpr int kMaxPartialBlocks = 2048;
constexpr int kVecBlocks = 148 * 4;   // grid of the streaming vector kernels
constexpr int kRedGroups = 24;        // block groups of the two-level batched reductions
constexpr int kVecThreads = 256;
constexpr double kEps64 = 2.220446049250313e-16;

// Scalars of one PCG solve, resident on the device.  Stop codes match
// include/acgpu.h (0 converged, 1 maxits, 2..7 stop reasons).
struct PcgState {
  // inputs
  double tol;
  double maxtime_s;
  long long maxits;
  int stag_test;
  int pad0;
  // PCG scalars (src/pcg.jl:256-445)
  double nb, rho, best_rho, bestnr, alpha, beta, nr, mean;
  double sum_abs_x, sum_abs_r, sum_abs_p, sum_abs_q, sum_abs_z;
  long long itcnt;
  int stag_count;
  int status;
  int done;
  int xcur, xnext, xbest;      // indices of the three x buffers
  unsigned long long t_start;  // %globaltimer at the start of the loop
  // mixed precision outer loop
  double scale;                // |r64| used to normalise the inner rhs
  double nb64;                 // |b - mean(b)|
  double nr_true;              // |b - L x| / |b| after the last correction
  double inner_tol;
  double tol_user;             // outer tolerance on the true residual
  double min_inner_tol;
  long long maxits_user;       // budget of inner iterations over all steps
  long long total_its;
  int outer_its, outer_done;
  int max_outer;
  int sweep_error;             // a bounded wait of a sync-free sweep gave up
  long long nvert;             // vertices of this system (graphs of a group)
  int entering;                // joined a running serving loop: this pass is its pre-loop step
  int pad1;
  double pq_dot;               // batched loop: p.q summed by the mat-vec
  unsigned int counter[16];    // last-block tickets of the reducing kernels
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---- reductions ------------------------------------------------------------

template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double* smem) {
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) smem[wid * NV + k] = v[k];
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      v[k] = lane < nw ? smem[lane * NV + k] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
  }
  __syncthreads();
}

// Deterministic grid reduction: every block stores its partial, the last
// block to arrive sums the partials in block order.  Returns true in the last
// block, where thread 0 holds the totals in v.
template <int NV>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double* partials, unsigned int* counter) {
  __shared__ double smem[32 * NV];
  __shared__ bool am_last;
  block_reduce<NV>(v, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[k * gridDim.x + blockIdx.x] = v[k];
    __threadfence();
    unsigned int t = atomicAdd(counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) s += __ldcg(&partials[k * gridDim.x + i]);
    v[k] = s;
  }
  block_reduce<NV>(v, smem);
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

// Sum over the VL lanes of an aligned lane group.
template <int VL, typename T>
__device__ __forceinline__ T group_sum(T x) {
#pragma unroll
  for (int o = VL / 2; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// ---- sparse kernels --------------------------------------------------------

// Programmatic dependent launch: the part of a kernel before pdl_wait() may
// overlap the previous kernel in the stream; it must read only data that no
// kernel since the last full (non-PDL) launch writes.  pdl_trigger() lets the
// next kernel start its own prologue.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Sum over the lanes of an aligned group of `width` lanes (width 4, 8 or 32).
template <typename T>
__device__ __forceinline__ T group_sum_w(T x, int width) {
  if (width == 32) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  } else {
    for (int o = width >> 1; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  }
  return x;
}

// One row / vertex per VL-lane group, U entries per lane in flight.
template <typename T, int VL>
__device__ __forceinline__ T row_dot(const int* __restrict__ ptr, const int* __restrict__ idx,
                                     const T* __restrict__ val, const T* x, int row, bool active, int lane) {
  constexpr int U = 4;
  T acc = T(0);
  if (active) {
    const int k1 = __ldg(&ptr[row + 1]);
    for (int k = __ldg(&ptr[row]) + lane; k < k1; k += VL * U) {
      int id[U];
      T c[U];
#pragma unroll
      for (int j = 0; j < U; ++j) {
        const int kk = k + j * VL;
        id[j] = kk < k1 ? __ldg(&idx[kk]) : -1;
        c[j] = kk < k1 ? __ldg(&val[kk]) : T(0);
      }
#pragma unroll
      for (int j = 0; j < U; ++j)
        if (id[j] >= 0) acc += c[j] * x[id[j]];
    }
  }
  return group_sum<VL>(acc);
}

// ---- LDLinv sweep, one wide level per launch ---------------------------------
//
// Vertices of a level are ordered by decreasing forward in-degree; the first
// `nw` of a forward level (in-degree > 32) get a whole warp each, the others
// share a warp four at a time (8 lanes each).  Each lane keeps 4 entries in
// flight.  The constant structure and the per-vertex aux value (r for the
// forward sweep, g for the backward one) are loaded before pdl_wait().
constexpr int kLevelThreads = 256;
constexpr int kLightLanes = 8;
constexpr int kEntryUnroll = 4;

template <typename T, bool kForward>
__global__ void __launch_bounds__(kLevelThreads) k_level(int v0, int v1, int nw, const int* __restrict__ ptr,
                                                         const int* __restrict__ idx, const T* __restrict__ coef,
                                                         const T* __restrict__ aux, const T* __restrict__ sfwd, T* vals,
                                                         const PcgState* st) {
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  int v, gl, gw;
  if (warp < nw) {
    v = v0 + warp;
    gl = lane;
    gw = 32;
  } else {
    v = v0 + nw + (warp - nw) * (32 / kLightLanes) + lane / kLightLanes;
    gl = lane & (kLightLanes - 1);
    gw = kLightLanes;
  }
  const bool active = v < v1;
  int k0 = 0, k1 = 0;
  if (active) {
    k0 = __ldg(&ptr[v]);
    k1 = __ldg(&ptr[v + 1]);
  }
  int id[kEntryUnroll];
  T c[kEntryUnroll];
#pragma unroll
  for (int j = 0; j < kEntryUnroll; ++j) {
    const int k = k0 + gl + j * gw;
    id[j] = k < k1 ? __ldg(&idx[k]) : -1;
    c[j] = k < k1 ? __ldg(&coef[k]) : T(0);
  }
  const T a = active ? __ldg(&aux[v]) : T(0);
  pdl_wait();
  pdl_trigger();
  if (st && st->done) return;
  T acc = T(0);
#pragma unroll
  for (int j = 0; j < kEntryUnroll; ++j)
    if (id[j] >= 0) acc += c[j] * vals[id[j]];
  for (int k = k0 + gl + kEntryUnroll * gw; k < k1; k += gw) acc += __ldg(&coef[k]) * vals[__ldg(&idx[k])];
  acc = group_sum_w(acc, gw);
  if (active && gl == 0) vals[v] = kForward ? a + acc : a * sfwd[v] + acc;
}

// ---- LDLinv sweep, a run of thin levels in one CTA ----------------------------
//
// The run covers levels [l0, l1) = vertices [V0, V1).  Their values live in
// shared memory for the whole run (and are written through to global memory
// for later kernels); values of vertices outside the run are final before the
// kernel starts and are read from global memory.  Groups of kThinLanes lanes
// take one vertex; the structure of the next level's first step is loaded
// into registers while the current level finishes, so a level costs one
// shared-memory gather and a block barrier.
constexpr int kThinThreads = 1024;
constexpr int kThinLanes = 4;
constexpr int kThinGroups = kThinThreads / kThinLanes;

template <typename T>
struct ThinPrefetch {
  int v, k0, k1;
  int id[kEntryUnroll];
  T c[kEntryUnroll];
  T a;
};

template <typename T>
__device__ __forceinline__ void thin_fetch(ThinPrefetch<T>& f, int v, int vend, const int* __restrict__ sptr, int V0,
                                          const int* __restrict__ idx, const T* __restrict__ coef,
                                          const T* __restrict__ aux, int gl) {
  f.v = v;
  f.k0 = f.k1 = 0;
  if (v < vend) {
    f.k0 = sptr[v - V0];
    f.k1 = sptr[v - V0 + 1];
    f.a = __ldg(&aux[v]);
  } else {
    f.a = T(0);
  }
#pragma unroll
  for (int j = 0; j < kEntryUnroll; ++j) {
    const int k = f.k0 + gl + j * kThinLanes;
    f.id[j] = k < f.k1 ? __ldg(&idx[k]) : -1;
    f.c[j] = k < f.k1 ? __ldg(&coef[k]) : T(0);
  }
}

template <typename T>
__device__ __forceinline__ T thin_value(int id, int V0, int V1, const T* sv, const T* vals) {
  return (id >= V0 && id < V1) ? sv[id - V0] : vals[id];
}

// Shared memory: values (NV of T), then row pointers of the run (NV+1 ints),
// then level offsets relative to V0 (L+1 ints).
template <typename T, bool kForward>
__global__ void __launch_bounds__(kThinThreads, 1) k_thin(int l0, int l1, const int* __restrict__ lvl_off,
                                                           const int* __restrict__ ptr, const int* __restrict__ idx,
                                                           const T* __restrict__ coef, const T* __restrict__ aux,
                                                           const T* __restrict__ sfwd, T* vals, const PcgState* st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int V0 = __ldg(&lvl_off[l0]), V1 = __ldg(&lvl_off[l1]);
  const int NV = V1 - V0, NL = l1 - l0;
  T* sv = reinterpret_cast<T*>(smem_raw);
  int* sptr = reinterpret_cast<int*>(sv + NV);
  int* soff = sptr + NV + 1;
  for (int i = threadIdx.x; i <= NV; i += blockDim.x) sptr[i] = __ldg(&ptr[V0 + i]);
  for (int i = threadIdx.x; i <= NL; i += blockDim.x) soff[i] = __ldg(&lvl_off[l0 + i]);
  pdl_wait();
  pdl_trigger();
  if (st && st->done) return;
  if (!kForward)
    for (int i = threadIdx.x; i < NV; i += blockDim.x) sv[i] = sfwd[V0 + i];
  __syncthreads();
  const int gl = threadIdx.x & (kThinLanes - 1);
  const int grp = threadIdx.x / kThinLanes;
  ThinPrefetch<T> f;
  {
    const int lf = kForward ? 0 : NL - 1;
    thin_fetch(f, soff[lf] + grp, soff[lf + 1], sptr, V0, idx, coef, aux, gl);
  }
  for (int step = 0; step < NL; ++step) {
    const int l = kForward ? step : NL - 1 - step;
    const int vs = soff[l], ve = soff[l + 1];
    for (int base = vs; base < ve; base += kThinGroups) {
      if (base != vs) thin_fetch(f, base + grp, ve, sptr, V0, idx, coef, aux, gl);
      const bool active = f.v < ve;
      T acc = T(0);
#pragma unroll
      for (int j = 0; j < kEntryUnroll; ++j)
        if (f.id[j] >= 0) acc += f.c[j] * thin_value(f.id[j], V0, V1, sv, vals);
      for (int k = f.k0 + gl + kEntryUnroll * kThinLanes; k < f.k1; k += kThinLanes)
        acc += __ldg(&coef[k]) * thin_value(__ldg(&idx[k]), V0, V1, sv, vals);
      acc = group_sum<kThinLanes>(acc);
      if (active && gl == 0) {
        const T out = kForward ? f.a + acc : f.a * sv[f.v - V0] + acc;
        sv[f.v - V0] = out;
        vals[f.v] = out;
      }
    }
    // prefetch the first step of the next level before the barrier
    if (step + 1 < NL) {
      const int ln = kForward ? step + 1 : NL - 2 - step;
      thin_fetch(f, soff[ln] + grp, soff[ln + 1], sptr, V0, idx, coef, aux, gl);
    }
    __syncthreads();
  }
}

// ---- LDLinv sweep, sync-free (one cooperative launch per sweep) -----------
//
// Every value of the sweep's output vector starts as a "pending" sentinel (a
// NaN with a payload arithmetic never produces); computing a vertex replaces
// it, so the value is its own ready flag.  Warps take tasks round-robin in
// level order (task t by warp t mod W); a task's inputs come from strictly
// earlier tasks, so with all warps co-resident (cooperative launch) the
// earliest unfinished task can always proceed.  Each wait polls the L2 copy
// with relaxed GPU-scope loads and gives up after spin_limit polls (a launch
// argument, kSpinLimit unless the solver's options set another), raising
// PcgState::sweep_error instead of hanging.
constexpr unsigned int kPendingF32 = 0x7fc0deadu;
constexpr unsigned long long kPendingF64 = 0x7ff8dead0000deadull;
constexpr unsigned int kSpinLimit = 1u << 22;
constexpr int kSweepThreads = 256;

__device__ __forceinline__ bool is_pending(float x) { return __float_as_uint(x) == kPendingF32; }
__device__ __forceinline__ bool is_pending(double x) {
  return (unsigned long long)__double_as_longlong(x) == kPendingF64;
}
template <typename T>
__device__ __forceinline__ T pending_value();
template <>
__device__ __forceinline__ float pending_value<float>() { return __uint_as_float(kPendingF32); }
template <>
__device__ __forceinline__ double pending_value<double>() { return __longlong_as_double((long long)kPendingF64); }

__device__ __forceinline__ float ld_relaxed(const float* p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ double ld_relaxed(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(float* p, float v) {
  asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// Poll until the value is no longer pending.  poll_mode 0: tight polls, then
// 64 ns sleeps; 1: tight polls only; 2: exponential backoff 32 ns .. 1 us.
template <typename T>
__device__ __noinline__ T wait_value_slow(const T* p, PcgState* st, int poll_mode, unsigned spin_limit) {
  unsigned int sleep_ns = 32;
  for (unsigned int spins = 1;; ++spins) {
    if (poll_mode == 0) {
      if (spins >= 64) __nanosleep(64);
    } else if (poll_mode == 2) {
      if (spins >= 4) {
        __nanosleep(sleep_ns);
        if (sleep_ns < 1024) sleep_ns <<= 1;
      }
    }
    const T x = ld_relaxed(p);
    if (!is_pending(x)) return x;
    if ((spins & 1023u) == 0 && *((volatile int*)&st->sweep_error)) return T(0);
    if (spins >= spin_limit) {
      atomicExch(&st->sweep_error, 1);
      return T(0);
    }
  }
}

template <typename T>
__device__ __forceinline__ T wait_value(const T* p, PcgState* st, int poll_mode, unsigned spin_limit) {
  const T x = ld_relaxed(p);
  return is_pending(x) ? wait_value_slow(p, st, poll_mode, spin_limit) : x;
}

// A task record (32 bytes): {first vertex, (count << 1) | heavy, p[0..4]} with
// p[i] = ptr[first + i], so a lane finds its entry range without another
// dependent load.  A heavy task is one vertex on 32 lanes, a light task up to
// 4 consecutive vertices of one level on 8 lanes each.
struct alignas(16) SweepTask {
  int v, cnt_heavy;
  int p[6];
};

template <typename T, int U = kEntryUnroll>
struct SweepEntries {
  int v, k0, k1, gw;
  bool active;
  int id[U];
  T c[U];
  T a, own;
};

__device__ __forceinline__ SweepTask load_task(const SweepTask* __restrict__ tasks, int t, int ntasks) {
  SweepTask r;
  if (t < ntasks) {
    const int4* q = reinterpret_cast<const int4*>(tasks + t);
    const int4 x = __ldg(q), y = __ldg(q + 1);
    r.v = x.x; r.cnt_heavy = x.y; r.p[0] = x.z; r.p[1] = x.w;
    r.p[2] = y.x; r.p[3] = y.y; r.p[4] = y.z; r.p[5] = y.w;
  } else {
    r.v = 0; r.cnt_heavy = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) r.p[i] = 0;
  }
  return r;
}

template <typename T, bool kForward, bool kLoadAux = true, int U = kEntryUnroll>
__device__ __forceinline__ void load_entries(SweepEntries<T, U>& e, const SweepTask& r, int lane,
                                             const int* __restrict__ idx, const T* __restrict__ coef,
                                             const T* __restrict__ aux, const T* __restrict__ sfwd, int vs = 1) {
  const bool heavy = r.cnt_heavy & 1;
  const int cnt = r.cnt_heavy >> 1;
  const int sub = heavy ? 0 : (lane >> 3);
  const int gw = heavy ? 32 : 8;
  const int gl = heavy ? lane : (lane & 7);
  e.active = sub < cnt;
  e.gw = gw;
  e.v = r.v + sub;
  int k0 = 0, k1 = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (i == sub) { k0 = r.p[i]; k1 = r.p[i + 1]; }
  if (!e.active) k0 = k1 = 0;
  e.k0 = k0 + gl;
  e.k1 = k1;
  e.a = (kLoadAux && e.active) ? __ldg(&aux[e.v]) : T(0);
  e.own = (kLoadAux && !kForward && e.active) ? __ldg(&sfwd[(size_t)e.v * vs]) : T(0);
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const int k = e.k0 + j * gw;
    e.id[j] = k < k1 ? __ldg(&idx[k]) : -1;
    e.c[j] = k < k1 ? __ldg(&coef[k]) : T(0);
  }
}

// Warp w runs tasks w, w+W, w+2W, ... (W warps in the grid).  Task records
// are loaded two tasks ahead and entries one task ahead, so only the waits on
// input values sit on the dependency chain.
template <typename T, bool kForward>
__global__ void __launch_bounds__(kSweepThreads) k_sweep(int ntasks, const SweepTask* __restrict__ tasks,
                                                         const int* __restrict__ idx, const T* __restrict__ coef,
                                                         const T* __restrict__ aux, const T* __restrict__ sfwd, T* out,
                                                         PcgState* st, int poll_mode, int vs,
                                                         unsigned spin_limit) {
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const int W = (int)((gridDim.x * blockDim.x) >> 5);
  int t = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  SweepTask r1 = load_task(tasks, t + W, ntasks);
  SweepEntries<T> e0;
  {
    const SweepTask r0 = load_task(tasks, t, ntasks);
    load_entries<T, kForward>(e0, r0, lane, idx, coef, aux, sfwd, vs);
  }
  for (; t < ntasks; t += W) {
    const SweepTask r2 = load_task(tasks, t + 2 * W, ntasks);
    SweepEntries<T> e1;
    load_entries<T, kForward>(e1, r1, lane, idx, coef, aux, sfwd, vs);
    const int gw = e0.gw;  // uniform across the warp: one task per warp
    T acc = T(0);
    // issue the loads of all prefetched entries before checking any of them
    T xv[kEntryUnroll];
#pragma unroll
    for (int j = 0; j < kEntryUnroll; ++j) xv[j] = e0.id[j] >= 0 ? ld_relaxed(&out[(size_t)e0.id[j] * vs]) : T(0);
    // FP32: inputs seen pending are polled again together (all polls of a
    // round in flight), not one wait after another; bounded like every wait.
    // Single-vector mixed solve on the 1M grid: 39.5 -> 36.9 ms.  FP64 keeps
    // the waits one by one: with joint polls, 256 graphs in one FP64 launch
    // (many graphs, thousands of tasks per level) went from 146.7 to 156.3 ms.
    unsigned pend = 0;
    if constexpr (sizeof(T) == 4) {
#pragma unroll
      for (int j = 0; j < kEntryUnroll; ++j)
        if (e0.id[j] >= 0 && is_pending(xv[j])) pend |= 1u << j;
    } else {
#pragma unroll
      for (int j = 0; j < kEntryUnroll; ++j)
        if (e0.id[j] >= 0 && is_pending(xv[j])) xv[j] = wait_value_slow(&out[(size_t)e0.id[j] * vs], st, poll_mode, spin_limit);
    }
    unsigned int sleep_ns = 32;
    for (unsigned int spins = 1; pend; ++spins) {
      if (poll_mode == 0) {
        if (spins >= 64) __nanosleep(64);
      } else if (poll_mode == 2) {
        if (spins >= 4) {
          __nanosleep(sleep_ns);
          if (sleep_ns < 1024) sleep_ns <<= 1;
        }
      }
#pragma unroll
      for (int j = 0; j < kEntryUnroll; ++j)
        if ((pend >> j) & 1u) xv[j] = ld_relaxed(&out[(size_t)e0.id[j] * vs]);
      unsigned still = 0;
#pragma unroll
      for (int j = 0; j < kEntryUnroll; ++j)
        if (((pend >> j) & 1u) && is_pending(xv[j])) still |= 1u << j;
      pend = still;
      if (pend && (((spins & 1023u) == 0 && *((volatile int*)&st->sweep_error)) || spins >= spin_limit)) {
        atomicExch(&st->sweep_error, 1);
#pragma unroll
        for (int j = 0; j < kEntryUnroll; ++j)
          if ((pend >> j) & 1u) xv[j] = T(0);
        break;
      }
    }
#pragma unroll
    for (int j = 0; j < kEntryUnroll; ++j)
      if (e0.id[j] >= 0) acc += e0.c[j] * xv[j];
    for (int k = e0.k0 + kEntryUnroll * gw; k < e0.k1; k += gw)
      acc += __ldg(&coef[k]) * wait_value(&out[(size_t)__ldg(&idx[k]) * vs], st, poll_mode, spin_limit);
    __syncwarp();  // reconverge after the divergent waits before the shuffles
    acc = group_sum_w(acc, gw);
    if (e0.active && (lane & (gw - 1)) == 0) st_relaxed(&out[(size_t)e0.v * vs], kForward ? e0.a + acc : e0.a * e0.own + acc);
    e0 = e1;
    r1 = r2;
  }
}

// ---- the narrow tail of the DAG in one CTA -----------------------------------
//
// The last NL levels (vertices [V0, V0+NV)) have at most 32 tasks each.  One
// 1024-thread CTA walks them level by level (forward: upwards, backward:
// downwards) with a block barrier between levels; the tail's values live in
// shared memory (and are written through to global memory), so a level costs
// a shared-memory gather and a barrier instead of a cross-SM hop.  Warp w runs
// task w of each level.  Task records are loaded two levels ahead and
// entries one level ahead.  lvl_tasks[i] = {first task, task count} of tail
// level i in the sweep's task table.
constexpr int kTailThreads = 1024;
constexpr int kTailWarps = kTailThreads / 32;

template <typename T, bool kForward>
__global__ void __launch_bounds__(kTailThreads, 1) k_tail(int NL, int V0, int NV, const int2* __restrict__ lvl_tasks,
                                                         int ntasks, const SweepTask* __restrict__ tasks,
                                                         const int* __restrict__ idx, const T* __restrict__ coef,
                                                         const T* __restrict__ aux, const T* __restrict__ sfwd,
                                                         T* out, const PcgState* st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sv = reinterpret_cast<T*>(smem_raw);
  int2* lt = reinterpret_cast<int2*>(sv + NV + (NV & 1));
  if (st && st->done) return;
  for (int i = threadIdx.x; i < NL; i += blockDim.x) lt[i] = lvl_tasks[i];
  if (!kForward)
    for (int i = threadIdx.x; i < NV; i += blockDim.x) sv[i] = __ldg(&sfwd[V0 + i]);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  auto task_of = [&](int step) -> int {
    if (step >= NL) return INT_MAX;
    const int2 r = lt[kForward ? step : NL - 1 - step];
    return w < r.y ? r.x + w : INT_MAX;
  };
  SweepTask r1 = load_task(tasks, task_of(1), ntasks);
  SweepEntries<T> e0;
  {
    const SweepTask r0 = load_task(tasks, task_of(0), ntasks);
    load_entries<T, kForward>(e0, r0, lane, idx, coef, aux, sfwd);
  }
  for (int step = 0; step < NL; ++step) {
    const SweepTask r2 = load_task(tasks, task_of(step + 2), ntasks);
    SweepEntries<T> e1;
    load_entries<T, kForward>(e1, r1, lane, idx, coef, aux, sfwd);
    const int2 cur = lt[kForward ? step : NL - 1 - step];
    // the first task of this warp came through the pipeline; further tasks of
    // a level (more than 32 of them is excluded by the host) never occur
    if (w < cur.y) {
      const int gw = e0.gw;
      T acc = T(0);
      T xv[kEntryUnroll];
#pragma unroll
      for (int j = 0; j < kEntryUnroll; ++j) {
        const int id = e0.id[j];
        xv[j] = id < 0 ? T(0) : (id >= V0 ? sv[id - V0] : out[id]);
      }
#pragma unroll
      for (int j = 0; j < kEntryUnroll; ++j) acc += e0.c[j] * xv[j];
      for (int k = e0.k0 + kEntryUnroll * gw; k < e0.k1; k += gw) {
        const int id = __ldg(&idx[k]);
        acc += __ldg(&coef[k]) * (id >= V0 ? sv[id - V0] : out[id]);
      }
      acc = group_sum_w(acc, gw);
      if (e0.active && (lane & (gw - 1)) == 0) {
        const T res = kForward ? e0.a + acc : e0.a * e0.own + acc;
        sv[e0.v - V0] = res;
        out[e0.v] = res;
      }
    }
    __syncthreads();
    e0 = e1;
    r1 = r2;
  }
}

template <typename T>
constexpr size_t tail_smem_bytes(int nv, int nl) {
  return (size_t)(nv + (nv & 1)) * sizeof(T) + (size_t)nl * sizeof(int2);
}

template <typename T>
__global__ void k_fill_pending(int n, T* a, T* b, int vs = 1) {
  const T pv = pending_value<T>();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    a[(size_t)i * vs] = pv;
    if (b) b[(size_t)i * vs] = pv;
  }
}

// Shared memory bytes of a thin run with nv vertices and nl levels.
template <typename T>
constexpr size_t thin_smem_bytes(int nv, int nl) {
  return (size_t)nv * sizeof(T) + (size_t)(nv + 1) * sizeof(int) + (size_t)(nl + 1) * sizeof(int);
}

}  // namespace acg
