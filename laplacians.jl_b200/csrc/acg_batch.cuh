// Batched solves: k right-hand sides of one graph in the same kernels.
//
// Vectors are vertex-major blocks n x kp (kp = k rounded up to 8, 16, 32 or
// 64): element (v, c) at v*kp + c, so one vertex's kp values are contiguous
// and a sweep reads each factor entry once for all columns.  Padding columns
// carry a zero right-hand side and stop at set-up.  Every column is its own
// PCG system with its own PcgState (the same scalar logic as the
// one-right-hand-side kernels, run by thread c for column c); a launch ends
// early only when every column has stopped.
#pragma once
#include <type_traits>

#include "acg_pcg.cuh"

namespace acg {

constexpr int kMaxBatch = 64;
// launch shape of the per-iteration batched vector kernels: 2 blocks of 512
// threads per SM, each thread keeping four elements' loads in flight
constexpr int kBVecThreads = 512;
constexpr int kBVecBlocks = 148 * 2;
constexpr int kBatchLanes = 8;  // lanes per vertex in the batched sweeps and mat-vec
// Rounds of a task's entries the batched sweeps prefetch with the task.  At
// the default heavy threshold of 8 a light task's vertices have at most 8
// entries (one round on 8 lanes) and a heavy task's one round covers 32;
// longer rows load their later rounds as they go.  One round instead of four
// frees the registers that spilled at two blocks per SM (140 -> 52 B per
// thread at 64 FP32 columns; forward 0.895 -> 0.834 ms, backward 1.036 ->
// 0.977 ms on the 1M grid).
constexpr int kBatchEntryUnroll = 1;

struct BatchShared {
  int all_done;     // every column stopped
  int sweep_error;  // a bounded sweep wait gave up
  int k;            // right-hand sides in this launch (the rest of kp is padding)
  int l1_due;       // kb_yzr deferred the third L1 test of some column to kb_pupdate_z
  int pq_full;      // kb_pq makes its pass: some column's next step runs the L1 tests
  int pad;
  unsigned int counter[16];
  unsigned int gcounter[16][kRedGroups];  // per-group tickets of the two-level reductions
};

// ---- vector relaxed loads/stores of CPL consecutive values -----------------

template <typename T, int CPL>
struct Row {
  T v[CPL];
};

template <typename T, int CPL>
__device__ __forceinline__ void ld_row(Row<T, CPL>& r, const T* p) {
#pragma unroll
  for (int j = 0; j < CPL; ++j) r.v[j] = ld_relaxed(p + j);
}

template <int CPL>
__device__ __forceinline__ void ld_row(Row<float, CPL>& r, const float* p) {
  if constexpr (CPL % 4 == 0) {
#pragma unroll
    for (int q = 0; q < CPL / 4; ++q)
      asm volatile("ld.relaxed.gpu.global.v4.f32 {%0,%1,%2,%3}, [%4];"
                   : "=f"(r.v[4 * q]), "=f"(r.v[4 * q + 1]), "=f"(r.v[4 * q + 2]), "=f"(r.v[4 * q + 3])
                   : "l"(p + 4 * q)
                   : "memory");
  } else {
#pragma unroll
    for (int j = 0; j < CPL; ++j) r.v[j] = ld_relaxed(p + j);
  }
}

template <int CPL>
__device__ __forceinline__ void ld_row(Row<double, CPL>& r, const double* p) {
  if constexpr (CPL % 2 == 0) {
#pragma unroll
    for (int q = 0; q < CPL / 2; ++q)
      asm volatile("ld.relaxed.gpu.global.v2.f64 {%0,%1}, [%2];"
                   : "=d"(r.v[2 * q]), "=d"(r.v[2 * q + 1])
                   : "l"(p + 2 * q)
                   : "memory");
  } else {
#pragma unroll
    for (int j = 0; j < CPL; ++j) r.v[j] = ld_relaxed(p + j);
  }
}

template <typename T, int CPL>
__device__ __forceinline__ bool row_pending(const Row<T, CPL>& r) {
  bool any = false;
#pragma unroll
  for (int j = 0; j < CPL; ++j) any |= is_pending(r.v[j]);
  return any;
}

template <int CPL>
__device__ __forceinline__ void st_row(float* p, const float (&v)[CPL]) {
  if constexpr (CPL % 4 == 0) {
#pragma unroll
    for (int q = 0; q < CPL / 4; ++q)
      asm volatile("st.relaxed.gpu.global.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(p + 4 * q), "f"(v[4 * q]),
                   "f"(v[4 * q + 1]), "f"(v[4 * q + 2]), "f"(v[4 * q + 3])
                   : "memory");
  } else {
#pragma unroll
    for (int j = 0; j < CPL; ++j) st_relaxed(p + j, v[j]);
  }
}
template <int CPL>
__device__ __forceinline__ void st_row(double* p, const double (&v)[CPL]) {
  if constexpr (CPL % 2 == 0) {
#pragma unroll
    for (int q = 0; q < CPL / 2; ++q)
      asm volatile("st.relaxed.gpu.global.v2.f64 [%0], {%1,%2};" ::"l"(p + 2 * q), "d"(v[2 * q]), "d"(v[2 * q + 1])
                   : "memory");
  } else {
#pragma unroll
    for (int j = 0; j < CPL; ++j) st_relaxed(p + j, v[j]);
  }
}

// Streaming accesses (read or written once per launch) go through L2 with an
// evict-first policy, so that they do not push out rows that are gathered
// several times: in the batched sweeps the right-hand-side row a task reads
// and the pending mark it writes (the output rows stay, for the successors'
// gathers), in the batched mat-vec the rows of q (p's rows stay, for the
// neighbours' gathers).  Measured on the 1M grid at 64 columns: forward /
// backward sweep 0.836 / 0.980 -> 0.831 / 0.956 ms, mat-vec 0.263 -> 0.243
// ms, 571.5 -> 579.7 solves/s.
__device__ __forceinline__ unsigned long long l2_evict_first_policy() {
  unsigned long long pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
template <int CPL>
__device__ __forceinline__ void ld_stream_row(float (&v)[CPL], const float* p, unsigned long long pol) {
  if constexpr (CPL % 4 == 0) {
#pragma unroll
    for (int q = 0; q < CPL / 4; ++q)
      asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
          : "=f"(v[4 * q]), "=f"(v[4 * q + 1]), "=f"(v[4 * q + 2]), "=f"(v[4 * q + 3])
          : "l"(p + 4 * q), "l"(pol));
  } else {
#pragma unroll
    for (int j = 0; j < CPL; ++j) v[j] = __ldg(p + j);
  }
}
template <int CPL>
__device__ __forceinline__ void ld_stream_row(double (&v)[CPL], const double* p, unsigned long long pol) {
  if constexpr (CPL % 2 == 0) {
#pragma unroll
    for (int q = 0; q < CPL / 2; ++q)
      asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0,%1}, [%2], %3;"
          : "=d"(v[2 * q]), "=d"(v[2 * q + 1])
          : "l"(p + 2 * q), "l"(pol));
  } else {
#pragma unroll
    for (int j = 0; j < CPL; ++j) v[j] = __ldg(p + j);
  }
}
template <int CPL>
__device__ __forceinline__ void st_stream_row(float* p, const float (&v)[CPL], unsigned long long pol) {
  if constexpr (CPL % 4 == 0) {
#pragma unroll
    for (int q = 0; q < CPL / 4; ++q)
      asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1,%2,%3,%4}, %5;" ::"l"(p + 4 * q), "f"(v[4 * q]),
                   "f"(v[4 * q + 1]), "f"(v[4 * q + 2]), "f"(v[4 * q + 3]), "l"(pol)
                   : "memory");
  } else {
    st_row<CPL>(p, v);
  }
}
template <int CPL>
__device__ __forceinline__ void st_stream_row(double* p, const double (&v)[CPL], unsigned long long pol) {
  if constexpr (CPL % 2 == 0) {
#pragma unroll
    for (int q = 0; q < CPL / 2; ++q)
      asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1,%2}, %3;" ::"l"(p + 2 * q), "d"(v[2 * q]),
                   "d"(v[2 * q + 1]), "l"(pol)
                   : "memory");
  } else {
    st_row<CPL>(p, v);
  }
}

// Build-time tuning of the batched sweeps: resident blocks per SM the 32- and
// 64-column FP32 sweeps are compiled for (their register budget), and the
// input rows a lane loads per batch (rows of at most 32 bytes, wider rows).
#ifndef ACG_BSWEEP_F32_BLOCKS
#define ACG_BSWEEP_F32_BLOCKS 2
#endif
#ifndef ACG_BSWEEP_ROWS
#define ACG_BSWEEP_ROWS 8
#endif
#ifndef ACG_BSWEEP_WIDE_ROWS  // the same for rows wider than 32 bytes
#define ACG_BSWEEP_WIDE_ROWS 8
#endif

// ---- batched sync-free sweep -----------------------------------------------
//
// Task records as in k_sweep.  Groups of 8 lanes; lane l of a group owns
// columns [l*CPL, (l+1)*CPL).  A light task puts one vertex on each group;
// a heavy task puts its one vertex on all four groups, group g taking the
// entries 8g..8g+7 of every round of 32, and the four partial sums are
// combined with shuffles.  In round j lane l of a group holds entry
// gl + j*gw of the vertex (the first kBatchEntryUnroll rounds are prefetched
// with the task), broadcasts it to its group, and the group loads the input rows in
// batches of EB with every load issued before any is checked.
//
// Blocks per SM the register budget is fitted to.  The FP32 sweeps of 32 and
// 64 columns are held to 128 registers so that two blocks share an SM: their
// wide levels are bound by how many tasks are in flight, and twice the warps
// outweigh the few spilled registers (measured on the 1M grid, 64 columns:
// forward 1.05 -> 0.90 ms, backward 1.24 -> 1.04 ms, with 140-148 B of
// spills; loading 4 rows per batch instead of 8 to avoid the spills was
// slower, 1.08 / 1.10 ms; 32 columns: 0.90 / 0.95 -> 0.66 / 0.78 ms, no
// spills).  The narrower FP32 sweeps fit two blocks anyway.  Three blocks
// (80 registers, 4-row batches) were slower again: 1.21 / 1.25 ms.  The
// 64-column FP64 sweeps run one block per SM and load 8 of their 64-byte rows
// per batch (242 registers, no spills; 4 rows: 1.87 / 1.78 -> 1.42 / 1.39 ms).
template <typename T, int CPL>
__host__ __device__ constexpr int kb_sweep_min_blocks() {
  return (sizeof(T) == 4 && CPL >= 4) ? ACG_BSWEEP_F32_BLOCKS : 1;
}

template <typename T, int CPL, bool kForward>
__global__ void __launch_bounds__(kSweepThreads, kb_sweep_min_blocks<T, CPL>())
    kb_sweep(int ntasks, const SweepTask* __restrict__ tasks, const int* __restrict__ idx,
             const T* __restrict__ coef, const T* __restrict__ aux, const T* sfwd, T* out, T* mark,
             BatchShared* bs, unsigned spin_limit) {
  if (bs->all_done) return;
  constexpr int kp = CPL * kBatchLanes;
  // rows loaded per batch: a whole slot of 8 entries where registers allow
  constexpr int EB = (CPL * sizeof(T) <= 32) ? ACG_BSWEEP_ROWS : ACG_BSWEEP_WIDE_ROWS;
  const int lane = threadIdx.x & 31;
  const int gl = lane & 7;
  const int W = (int)((gridDim.x * blockDim.x) >> 5);
  int t = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const unsigned long long pol = l2_evict_first_policy();
  SweepTask r1 = load_task(tasks, t + W, ntasks);
  SweepEntries<T, kBatchEntryUnroll> e0;
  {
    const SweepTask r0 = load_task(tasks, t, ntasks);
    load_entries<T, true, false, kBatchEntryUnroll>(e0, r0, lane, idx, coef, coef, coef);
  }
  for (; t < ntasks; t += W) {
    const SweepTask r2 = load_task(tasks, t + 2 * W, ntasks);
    SweepEntries<T, kBatchEntryUnroll> e1;
    load_entries<T, true, false, kBatchEntryUnroll>(e1, r1, lane, idx, coef, coef, coef);
    const int gw = e0.gw;  // 32 for a heavy task, 8 for a light one (uniform per warp)
    const int k0 = e0.k0 - (gw == 32 ? lane : gl);  // first entry of this lane's vertex
    T acc[CPL];
#pragma unroll
    for (int j = 0; j < CPL; ++j) acc[j] = T(0);
    Row<T, CPL> a;
    if (e0.active && (gw == 8 || lane < 8)) {
      if (kForward) {
        ld_stream_row<CPL>(a.v, aux + (size_t)e0.v * kp + gl * CPL, pol);
      } else {
        ld_stream_row<CPL>(a.v, sfwd + (size_t)e0.v * kp + gl * CPL, pol);
        const T g = __ldg(&aux[e0.v]);
#pragma unroll
        for (int j = 0; j < CPL; ++j) a.v[j] = g * a.v[j];
      }
    }
    int rounds = e0.active ? (e0.k1 - k0 + gw - 1) / gw : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rounds = max(rounds, __shfl_xor_sync(0xffffffffu, rounds, o));
    for (int j = 0; j < rounds; ++j) {
      int myid;
      T myc;
      if (j < kBatchEntryUnroll) {
        myid = e0.id[0];
        myc = e0.c[0];
#pragma unroll
        for (int q = 1; q < kBatchEntryUnroll; ++q)
          if (q == j) {
            myid = e0.id[q];
            myc = e0.c[q];
          }
      } else {
        const int k = e0.k0 + j * gw;
        myid = (e0.active && k < e0.k1) ? __ldg(&idx[k]) : -1;
        myc = (e0.active && k < e0.k1) ? __ldg(&coef[k]) : T(0);
      }
#pragma unroll
      for (int l0 = 0; l0 < 8; l0 += EB) {
        Row<T, CPL> vals[EB];
        T cs[EB];
        int ids[EB];
#pragma unroll
        for (int u = 0; u < EB; ++u) {
          ids[u] = __shfl_sync(0xffffffffu, myid, (lane & ~7) | (l0 + u));
          cs[u] = __shfl_sync(0xffffffffu, myc, (lane & ~7) | (l0 + u));
        }
#pragma unroll
        for (int u = 0; u < EB; ++u)
          if (ids[u] >= 0) ld_row<CPL>(vals[u], out + (size_t)ids[u] * kp + gl * CPL);
        unsigned pend = 0;
#pragma unroll
        for (int u = 0; u < EB; ++u)
          if (ids[u] >= 0 && row_pending(vals[u])) pend |= 1u << u;
        // Rows seen pending are polled again together, every poll of a round
        // in flight at once, until none is pending.  Waiting for them one at
        // a time paid a full L2 round trip for each stale row even when it
        // had become ready during the earlier waits (measured on the 1M grid
        // at 64 columns: backward 0.953 -> 0.823 ms, forward 0.816 -> 0.789
        // ms).  A row read ready is final: rows are written once per sweep.
        // The wait is bounded: after spin_limit rounds, or once another wait
        // has given up, the sweep error is raised and the rows still pending
        // read as zeros.
        for (unsigned int spins = 1; pend; ++spins) {
          if (spins >= 64) __nanosleep(64);
#pragma unroll
          for (int u = 0; u < EB; ++u)
            if ((pend >> u) & 1u) ld_row<CPL>(vals[u], out + (size_t)ids[u] * kp + gl * CPL);
          unsigned still = 0;
#pragma unroll
          for (int u = 0; u < EB; ++u)
            if (((pend >> u) & 1u) && row_pending(vals[u])) still |= 1u << u;
          pend = still;
          if (pend && (((spins & 1023u) == 0 && *((volatile int*)&bs->sweep_error)) || spins >= spin_limit)) {
            atomicExch(&bs->sweep_error, 1);
#pragma unroll
            for (int u = 0; u < EB; ++u)
              if ((pend >> u) & 1u) {
#pragma unroll
                for (int q = 0; q < CPL; ++q) vals[u].v[q] = T(0);
              }
            break;
          }
        }
#pragma unroll
        for (int u = 0; u < EB; ++u) {
          if (ids[u] < 0) continue;
#pragma unroll
          for (int q = 0; q < CPL; ++q) acc[q] += cs[u] * vals[u].v[q];
        }
      }
      // Reconverge explicitly after the (divergent, sleeping) waits: without
      // it the next shuffle waits for the lanes that skipped the wait far
      // longer than the wait itself (measured: 2.9 us instead of 0.9 us per
      // dependency hop at 64 columns).
      __syncwarp();
    }
    if (gw == 32) {  // combine the four groups of a heavy task
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], 8);
        acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], 16);
      }
    }
    if (e0.active && (gw == 8 || lane < 8)) {
      T res[CPL];
#pragma unroll
      for (int q = 0; q < CPL; ++q) res[q] = a.v[q] + acc[q];
      st_row<CPL>(out + (size_t)e0.v * kp + gl * CPL, res);
      if (mark) {
        // the vertex's row of the other sweep's vector is dead from here on
        // (forward: y, read by no one until the backward rewrites it;
        // backward: s, whose only reader was this task): mark it pending
        // for the next sweep instead of a separate pass over the vector
#pragma unroll
        for (int q = 0; q < CPL; ++q) res[q] = pending_value<T>();
        st_stream_row<CPL>(mark + (size_t)e0.v * kp + gl * CPL, res, pol);
      }
    }
    e0 = e1;
    r1 = r2;
  }
}

// ---- batched mat-vec: q = L p for kp columns -------------------------------

// A lane's slice of a row through the read-only path (p does not change
// during the mat-vec), in 16-byte pieces where the slice allows.
template <typename T, int CPL>
__device__ __forceinline__ void ldg_row(T (&v)[CPL], const T* src) {
  if constexpr (sizeof(T) == 4 && CPL % 4 == 0) {
#pragma unroll
    for (int q = 0; q < CPL / 4; ++q) {
      const float4 x = __ldg(reinterpret_cast<const float4*>(src) + q);
      v[4 * q] = x.x;
      v[4 * q + 1] = x.y;
      v[4 * q + 2] = x.z;
      v[4 * q + 3] = x.w;
    }
  } else if constexpr (sizeof(T) == 8 && CPL % 2 == 0) {
#pragma unroll
    for (int q = 0; q < CPL / 2; ++q) {
      const double2 x = __ldg(reinterpret_cast<const double2*>(src) + q);
      v[2 * q] = x.x;
      v[2 * q + 1] = x.y;
    }
  } else {
#pragma unroll
    for (int q = 0; q < CPL; ++q) v[q] = __ldg(src + q);
  }
}

template <int NV, int VPT>
__device__ __forceinline__ bool batch_reduce_v(double (&v)[NV][VPT], int kp, double* partials, BatchShared* bs,
                                               int ci, double (&out)[NV]);

// One row per group of 8 lanes.  The group's lanes load up to 8 of the row's
// entries at once, share them with shuffles inside the group, and issue every
// gathered row before the first multiply-add; entries are summed in row order.
//
// kDot (the PCG loop body): also p.q per column, each lane summing its rows'
// p_v * q_v (p_v read again, from L1: the row's diagonal entry gathered it), in
// FP32 for FP32 vectors and FP64 for FP64, then over the grid in FP64 in a
// fixed order (st[c].pq_dot).  The last block also tells kb_pq whether some
// column's next step is one of the every-10th steps that need |p|_1 and |q|_1
// (BatchShared::pq_full); on the other steps kb_pq skips its pass over p and q.
template <typename T, int CPL, bool kDot = false>
__global__ void __launch_bounds__(kVecThreads) kb_spmv(int n, const int* __restrict__ ptr, const int* __restrict__ idx,
                                                       const T* __restrict__ val, const T* __restrict__ p,
                                                       T* __restrict__ q, BatchShared* bs, PcgState* st = nullptr,
                                                       double* partials = nullptr) {
  if (bs && bs->all_done) return;
  constexpr int kp = CPL * kBatchLanes;
  using Acc = typename std::conditional<sizeof(T) == 4, float, double>::type;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int gl = gt & 7;
  const unsigned gmask = 0xffu << (threadIdx.x & 24);  // this group's lanes
  const int groups = gridDim.x * blockDim.x / 8;
  const unsigned long long pol = l2_evict_first_policy();
  Acc pq[CPL];
#pragma unroll
  for (int j = 0; j < CPL; ++j) pq[j] = Acc(0);
  int row = gt / 8;
  int n0 = row < n ? __ldg(&ptr[row]) : 0, n1 = row < n ? __ldg(&ptr[row + 1]) : 0;
  for (; row < n; row += groups) {
    const int k0 = n0, k1 = n1;
    // the group's next row: its extent is loaded while this row is summed
    const int nxt = row + groups;
    n0 = nxt < n ? __ldg(&ptr[nxt]) : 0;
    n1 = nxt < n ? __ldg(&ptr[nxt + 1]) : 0;
    T acc[CPL];
#pragma unroll
    for (int j = 0; j < CPL; ++j) acc[j] = T(0);
    for (int kb = k0; kb < k1; kb += 8) {
      const int k = kb + gl;
      const int myid = k < k1 ? __ldg(&idx[k]) : -1;
      const T myc = k < k1 ? __ldg(&val[k]) : T(0);
      int ids[8];
      T cs[8];
      T v[8][CPL];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        ids[u] = __shfl_sync(gmask, myid, u, 8);
        cs[u] = __shfl_sync(gmask, myc, u, 8);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (ids[u] >= 0) ldg_row<T, CPL>(v[u], p + (size_t)ids[u] * kp + gl * CPL);
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (ids[u] >= 0) {
#pragma unroll
          for (int j = 0; j < CPL; ++j) acc[j] += cs[u] * v[u][j];
        }
    }
    st_stream_row<CPL>(q + (size_t)row * kp + gl * CPL, acc, pol);
    if constexpr (kDot) {
      T own[CPL];
      ldg_row<T, CPL>(own, p + (size_t)row * kp + gl * CPL);
#pragma unroll
      for (int j = 0; j < CPL; ++j) pq[j] += (Acc)own[j] * (Acc)acc[j];
    }
  }
  if constexpr (kDot) {
    double v[1][CPL];
#pragma unroll
    for (int j = 0; j < CPL; ++j) v[0][j] = (double)pq[j];
    double tot[1];
    if (batch_reduce_v<1, CPL>(v, kp, partials, bs, 13, tot)) {
      const int c = threadIdx.x;
      bool need = false;
      if (c < kp) {
        st[c].pq_dot = tot[0];
        need = !st[c].done && !st[c].entering && (st[c].itcnt + 1) % 10 == 0;
      }
      const int any = __syncthreads_or(need);
      if (threadIdx.x == 0) bs->pq_full = any;
    }
  }
}

// ---- per-column reductions ---------------------------------------------------
//
// Element i = v*kp + c is visited by threads of a fixed column (blockDim and
// the grid stride are multiples of kp).  Block sums per column go through
// shared memory in thread order, partials per (block, column) are summed by
// the last block in block order: deterministic for a given n and kp.

template <int NV>
__device__ __forceinline__ bool batch_reduce(double (&v)[NV], int kp, double* partials, unsigned int* counter,
                                             double (&out)[NV]) {
  __shared__ double sm[NV][kBVecThreads];
  __shared__ bool am_last;
#pragma unroll
  for (int q = 0; q < NV; ++q) sm[q][threadIdx.x] = v[q];
  __syncthreads();
  const int per = blockDim.x / kp;
  if ((int)threadIdx.x < kp) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int j = 0; j < per; ++j) s += sm[q][threadIdx.x + j * kp];
      partials[((size_t)q * gridDim.x + blockIdx.x) * kp + threadIdx.x] = s;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  // The last block: thread t sums, in block order, the partials of column
  // t % kp from a fixed contiguous range of blocks (part t / kp of `per`);
  // then the parts are added in order.  The shape depends only on the launch.
  {
    const int c = threadIdx.x % kp, part = threadIdx.x / kp;
    const int G = gridDim.x;
    const int b0 = (int)((long long)G * part / per), b1 = (int)((long long)G * (part + 1) / per);
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const double* pq = partials + (size_t)q * G * kp + c;
      double s = 0.0;
      int b = b0;
      for (; b + 8 <= b1; b += 8) {
        double l[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) l[u] = __ldcg(pq + (size_t)(b + u) * kp);
#pragma unroll
        for (int u = 0; u < 8; ++u) s += l[u];
      }
      for (; b < b1; ++b) s += __ldcg(pq + (size_t)b * kp);
      sm[q][threadIdx.x] = s;
    }
  }
  __syncthreads();
  if ((int)threadIdx.x < kp) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int j = 0; j < per; ++j) s += sm[q][threadIdx.x + j * kp];
      out[q] = s;
    }
  }
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

// Thread (c, part) of a block sums column c of NV tables over rows [r0, r1)
// (src[q * qstride + row * kp + c]), each table's rows in ascending order, with
// up to 8 loads in flight across the tables.
template <int NV>
__device__ __forceinline__ void sum_rows(const double* src, size_t qstride, int kp, int c, int r0, int r1,
                                         double (&s)[NV]) {
#pragma unroll
  for (int q = 0; q < NV; ++q) s[q] = 0.0;
  const int nr = r1 - r0, m = NV * nr;
  for (int j0 = 0; j0 < m; j0 += 8) {
    double l[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int j = j0 + u;
      l[u] = j < m ? __ldcg(src + (size_t)(j / nr) * qstride + (size_t)(r0 + j % nr) * kp + c) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int j = j0 + u;
#pragma unroll
      for (int q = 0; q < NV; ++q)
        if (j < m && j / nr == q) s[q] += l[u];
    }
  }
}

// Sums, per column, the rows [0, rows) of NV tables of kp columns into `out`
// of the threads below kp: the block's threads split the rows into
// blockDim / kp contiguous parts, and the parts are added in order.
template <int NV, int kTile>
__device__ __forceinline__ void block_sum_rows(const double* src, size_t qstride, int kp, int rows,
                                               double (&sm)[NV][kVecThreads * kTile], double (&out)[NV]) {
  const int per = (int)blockDim.x / kp;
  const int c = threadIdx.x % kp, part = threadIdx.x / kp;
  double s[NV];
  sum_rows<NV>(src, qstride, kp, c, (int)((long long)rows * part / per), (int)((long long)rows * (part + 1) / per), s);
#pragma unroll
  for (int q = 0; q < NV; ++q) sm[q][threadIdx.x] = s[q];
  __syncthreads();
  if ((int)threadIdx.x < kp) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double t = 0.0;
      for (int j = 0; j < per; ++j) t += sm[q][threadIdx.x + j * kp];
      out[q] = t;
    }
  }
}

// The same reduction when each thread holds VPT consecutive columns
// (v[q][j] for column (VPT * threadIdx.x + j) mod kp; blockDim * VPT and the
// grid stride are multiples of kp), in two levels: the block's values are laid
// out as VPT * blockDim virtual threads in shared memory and summed per column
// into one row of partials per block; the last block to finish in each of up
// to kRedGroups contiguous groups of blocks sums its group's rows into a group
// row, and the last group to finish sums the group rows.  One block alone
// would read every block's row (592 x NV x kp values) with a few loads in
// flight per thread, tens of dependent L2 round trips; two levels take a
// handful.  The order of every sum is fixed by the grid, so results repeat
// bit for bit.  Threads below kp of the returning block get the totals of
// column threadIdx.x in out.  partials holds NV * (gridDim + kRedGroups) * kp
// values.
template <int NV, int VPT>
__device__ __forceinline__ bool batch_reduce_v(double (&v)[NV][VPT], int kp, double* partials, BatchShared* bs,
                                               int ci, double (&out)[NV]) {
  constexpr int kTile = VPT > 4 ? VPT : 4;
  __shared__ double sm[NV][kVecThreads * kTile];
  __shared__ bool am_last;
#pragma unroll
  for (int q = 0; q < NV; ++q)
#pragma unroll
    for (int j = 0; j < VPT; ++j) sm[q][threadIdx.x * VPT + j] = v[q][j];
  __syncthreads();
  const int G = gridDim.x;
  const int gs = (G + kRedGroups - 1) / kRedGroups;  // blocks per group
  const int NG = (G + gs - 1) / gs;                   // groups
  const int g = blockIdx.x / gs, gb0 = g * gs, gb1 = min(G, gb0 + gs);
  double* grows = partials + (size_t)NV * G * kp;     // group rows: [q][NG][kp]
  const int per_v = (int)blockDim.x * VPT / kp;
  if ((int)threadIdx.x < kp) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int j = 0; j < per_v; ++j) s += sm[q][threadIdx.x + j * kp];
      partials[((size_t)q * G + blockIdx.x) * kp + threadIdx.x] = s;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    am_last = atomicAdd(&bs->gcounter[ci][g], 1u) == (unsigned)(gb1 - gb0 - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  // the group's last block: its rows into the group row
  {
    double t[NV];
    block_sum_rows<NV, kTile>(partials + (size_t)gb0 * kp, (size_t)G * kp, kp, gb1 - gb0, sm, t);
    if ((int)threadIdx.x < kp) {
#pragma unroll
      for (int q = 0; q < NV; ++q) grows[((size_t)q * NG + g) * kp + threadIdx.x] = t[q];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    bs->gcounter[ci][g] = 0u;
    __threadfence();
    am_last = atomicAdd(&bs->counter[ci], 1u) == (unsigned)(NG - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  block_sum_rows<NV, kTile>(grows, (size_t)NG * kp, kp, NG, sm, out);
  if (threadIdx.x == 0) bs->counter[ci] = 0u;
  return true;
}

// 16-byte vectors of the loop-body kernels: 4 FP32 or 2 FP64 columns.
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  static constexpr int W = 4;
  using V = float4;
  __device__ static void split(const V& x, float (&o)[4]) { o[0] = x.x; o[1] = x.y; o[2] = x.z; o[3] = x.w; }
  __device__ static V join(const float (&o)[4]) { return make_float4(o[0], o[1], o[2], o[3]); }
};
template <>
struct Vec16<double> {
  static constexpr int W = 2;
  using V = double2;
  __device__ static void split(const V& x, double (&o)[2]) { o[0] = x.x; o[1] = x.y; }
  __device__ static V join(const double (&o)[2]) { return make_double2(o[0], o[1]); }
};

// After the per-column scalar steps: end the launch's loop when all columns stopped.
// kLoop = false: a copy that never sets the loop's condition (so holds no
// conditional-handle call), for the timing graphs: profilers refuse to measure
// kernels that can set a graph's conditional handle.
template <bool kLoop = true>
__device__ __forceinline__ void batch_check_all(PcgState* st, BatchShared* bs, int kp, const LoopCtl& ctl) {
  __syncthreads();
  if (threadIdx.x == 0) {
    bool all = true;
    for (int c = 0; c < kp; ++c) all &= (st[c].done != 0);
    if (all) {
      bs->all_done = 1;
      if constexpr (kLoop) clear_loop(ctl);
    }
  }
}

// The per-iteration kernels below walk their n*kp elements with a grid
// stride that is a multiple of kp (each thread keeps one column) and four
// strides per step, all loads issued before any arithmetic; per-thread sums
// still run in element order.
constexpr int kBU = 4;

// The loop-body kernels (kb_pq, kb_update, kb_yzr, kb_pupdate_z) move 16
// bytes per access: thread t owns the W = 16 / sizeof(T) consecutive columns
// starting at (W * t) mod kp, walks the block in W-wide vectors with a grid
// stride that is a multiple of kp, and keeps kBU vectors of every operand in
// flight.  With 4-byte accesses the same kernels moved 2.7-5.3 TB/s on the 1M
// grid at 64 columns.

// pq, |p|_1, |q|_1 per column -> alpha, stagnation tests 1 and 2
template <typename T, bool kLoop = true>
__global__ void __launch_bounds__(kVecThreads) kb_pq(int n, int kp, const T* __restrict__ p, const T* __restrict__ q,
                                                     PcgState* st, BatchShared* bs, double* partials, double eps,
                                                     LoopCtl ctl) {
  if (bs->all_done) return;
  if (!bs->pq_full) {
    // p.q came with the mat-vec and no column runs its L1 tests on this step
    // (they alone read |p|_1 and |q|_1): only the scalar step, in block 0
    if (blockIdx.x == 0) {
      const int c = threadIdx.x;
      if (c < kp && !st[c].done) pcg_scalar_pq(&st[c], st[c].pq_dot, 0.0, 0.0, eps);
      batch_check_all<kLoop>(st, bs, kp, ctl);
    }
    return;
  }
  using VT = Vec16<T>;
  constexpr int W = VT::W;
  using V = typename VT::V;
  const size_t NW = (size_t)n * kp / W;
  const size_t S = (size_t)gridDim.x * blockDim.x;
  size_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const V* pv4 = reinterpret_cast<const V*>(p);
  const V* qv4 = reinterpret_cast<const V*>(q);
  double acc[3][W];
#pragma unroll
  for (int j = 0; j < W; ++j) acc[0][j] = acc[1][j] = acc[2][j] = 0.0;
  for (; i + (kBU - 1) * S < NW; i += kBU * S) {
    V pv[kBU], qv[kBU];
#pragma unroll
    for (int u = 0; u < kBU; ++u) {
      pv[u] = pv4[i + u * S];
      qv[u] = qv4[i + u * S];
    }
#pragma unroll
    for (int u = 0; u < kBU; ++u) {
      T a[W], b[W];
      VT::split(pv[u], a);
      VT::split(qv[u], b);
#pragma unroll
      for (int j = 0; j < W; ++j) {
        acc[0][j] += (double)a[j] * (double)b[j];
        acc[1][j] += fabs((double)a[j]);
        acc[2][j] += fabs((double)b[j]);
      }
    }
  }
  for (; i < NW; i += S) {
    T a[W], b[W];
    VT::split(pv4[i], a);
    VT::split(qv4[i], b);
#pragma unroll
    for (int j = 0; j < W; ++j) {
      acc[0][j] += (double)a[j] * (double)b[j];
      acc[1][j] += fabs((double)a[j]);
      acc[2][j] += fabs((double)b[j]);
    }
  }
  double tot[3];
  if (batch_reduce_v<3, W>(acc, kp, partials, bs, 0, tot)) {
    const int c = threadIdx.x;
    if (c < kp && !st[c].done) pcg_scalar_pq(&st[c], tot[0], tot[1], tot[2], eps);
    batch_check_all<kLoop>(st, bs, kp, ctl);
  }
}

// The update holds three vectors and a column of x per step: two steps in
// flight keep it within the registers of three blocks per SM.
constexpr int kBUx = 2;

// x' = x + alpha p, r -= alpha q (active columns); |r|^2, |x'|_1, |r|_1.  The
// sweeps' vectors s and y are marked pending by the sweeps themselves.  Each
// column keeps its x in its own one of three buffers, so x moves one value at
// a time; a vector whose columns have all stopped is skipped.
template <typename T, bool kLoop = true>
__global__ void __launch_bounds__(kVecThreads) kb_update(int n, int kp, T* x3, const T* __restrict__ p,
                                                         const T* __restrict__ q, T* __restrict__ r, PcgState* st,
                                                         BatchShared* bs, double* partials, LoopCtl ctl) {
  if (bs->all_done) return;
  using VT = Vec16<T>;
  constexpr int W = VT::W;
  using V = typename VT::V;
  const size_t N = (size_t)n * kp;
  const size_t NW = N / W;
  const size_t S = (size_t)gridDim.x * blockDim.x;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c0 = (int)((i0 * W) % kp);
  double al[W];
  const T* xc[W];
  T* xn[W];
  bool any = false;
#pragma unroll
  for (int j = 0; j < W; ++j) {
    const PcgState* sc = &st[c0 + j];
    const bool act = !sc->done;
    any |= act;
    al[j] = act ? sc->alpha : 0.0;  // a stopped column keeps its vectors
    xc[j] = x3 + (size_t)sc->xcur * N;
    xn[j] = x3 + (size_t)sc->xnext * N;
  }
  const V* pv4 = reinterpret_cast<const V*>(p);
  const V* qv4 = reinterpret_cast<const V*>(q);
  V* rv4 = reinterpret_cast<V*>(r);
  double acc[3][W];
#pragma unroll
  for (int j = 0; j < W; ++j) acc[0][j] = acc[1][j] = acc[2][j] = 0.0;
  size_t i = any ? i0 : NW;
  for (; i + (kBUx - 1) * S < NW; i += kBUx * S) {
    V pv[kBUx], qv[kBUx], rv[kBUx];
    T xv[kBUx][W];
#pragma unroll
    for (int u = 0; u < kBUx; ++u) {
      pv[u] = pv4[i + u * S];
      qv[u] = qv4[i + u * S];
      rv[u] = rv4[i + u * S];
#pragma unroll
      for (int j = 0; j < W; ++j) xv[u][j] = xc[j][(i + u * S) * W + j];
    }
#pragma unroll
    for (int u = 0; u < kBUx; ++u) {
      T a[W], b[W], rr[W], rw[W];
      VT::split(pv[u], a);
      VT::split(qv[u], b);
      VT::split(rv[u], rr);
#pragma unroll
      for (int j = 0; j < W; ++j) {
        const T xw = (T)((double)xv[u][j] + al[j] * (double)a[j]);
        rw[j] = (T)((double)rr[j] + (-al[j]) * (double)b[j]);
        xn[j][(i + u * S) * W + j] = xw;
        acc[0][j] += (double)rw[j] * (double)rw[j];
        acc[1][j] += fabs((double)xw);
        acc[2][j] += fabs((double)rw[j]);
      }
      rv4[i + u * S] = VT::join(rw);
    }
  }
  for (; i < NW; i += S) {
    T a[W], b[W], rr[W], rw[W];
    VT::split(pv4[i], a);
    VT::split(qv4[i], b);
    VT::split(rv4[i], rr);
#pragma unroll
    for (int j = 0; j < W; ++j) {
      const T xw = (T)((double)xc[j][i * W + j] + al[j] * (double)a[j]);
      rw[j] = (T)((double)rr[j] + (-al[j]) * (double)b[j]);
      xn[j][i * W + j] = xw;
      acc[0][j] += (double)rw[j] * (double)rw[j];
      acc[1][j] += fabs((double)xw);
      acc[2][j] += fabs((double)rw[j]);
    }
    rv4[i] = VT::join(rw);
  }
  double tot[3];
  if (batch_reduce_v<3, W>(acc, kp, partials, bs, 1, tot)) {
    const int cc = threadIdx.x;
    if (cc < kp && !st[cc].done) pcg_scalar_update(&st[cc], tot[0], tot[1], tot[2]);
    batch_check_all<kLoop>(st, bs, kp, ctl);
  }
}

template <typename T>
__global__ void __launch_bounds__(kBVecThreads) kb_ysum(int n, int kp, const T* __restrict__ y, PcgState* st,
                                                        BatchShared* bs, double* partials, LoopCtl ctl) {
  if (bs->all_done) return;
  const size_t N = (size_t)n * kp;
  const size_t S = (size_t)gridDim.x * blockDim.x;
  size_t i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[1] = {0.0};
  for (; i + (kBUx - 1) * S < N; i += kBUx * S) {
    T yv[kBUx];
#pragma unroll
    for (int u = 0; u < kBUx; ++u) yv[u] = y[i + u * S];
#pragma unroll
    for (int u = 0; u < kBUx; ++u) acc[0] += (double)yv[u];
  }
  for (; i < N; i += S) acc[0] += (double)y[i];
  double tot[1];
  if (batch_reduce<1>(acc, kp, partials, &bs->counter[2], tot)) {
    const int c = threadIdx.x;
    if (c < kp) {
      st[c].mean = tot[0] / (double)n;
      if (bs->sweep_error && !st[c].done) mark_stop(&st[c], kSweepTimeout);
    }
    batch_check_all(st, bs, kp, ctl);
  }
}

// The pre-loop step of a batched solve (init 1 or 2, see pcg_scalar_zdot):
// z = y - mean (in place), p = z; rho = z.r, |z|_1
template <typename T>
__global__ void __launch_bounds__(kBVecThreads) kb_zdot(int n, int kp, T* __restrict__ yz, const T* __restrict__ r,
                                                        T* __restrict__ p, PcgState* st, BatchShared* bs,
                                                        double* partials, double eps, int init, LoopCtl ctl) {
  if (bs->all_done) return;
  const size_t N = (size_t)n * kp;
  const size_t S = (size_t)gridDim.x * blockDim.x;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  const double mu = st[c].mean;
  double acc[2] = {0.0, 0.0};
  size_t i = i0;
  for (; i + (kBUx - 1) * S < N; i += kBUx * S) {
    T yv[kBUx], rv[kBUx];
#pragma unroll
    for (int u = 0; u < kBUx; ++u) {
      yv[u] = yz[i + u * S];
      rv[u] = r[i + u * S];
    }
#pragma unroll
    for (int u = 0; u < kBUx; ++u) {
      const T z = (T)((double)yv[u] - mu);
      yz[i + u * S] = z;
      if (init) p[i + u * S] = z;
      acc[0] += (double)z * (double)rv[u];
      acc[1] += fabs((double)z);
    }
  }
  for (; i < N; i += S) {
    const T z = (T)((double)yz[i] - mu);
    yz[i] = z;
    if (init) p[i] = z;
    acc[0] += (double)z * (double)r[i];
    acc[1] += fabs((double)z);
  }
  double tot[2];
  if (batch_reduce<2>(acc, kp, partials, &bs->counter[3], tot)) {
    const int cc = threadIdx.x;
    if (cc < kp && !st[cc].done) pcg_scalar_zdot(&st[cc], tot[0], tot[1], eps, init);
    batch_check_all(st, bs, kp, ctl);
  }
}

// The loop body's tail in two passes instead of three (kb_ysum, kb_zdot,
// kb_pupdate).  z = y - mean is never stored: kb_yzr sums y, y.r and r per
// column in one pass over y and r, and rho = (y - mean).r is y.r - mean * r.1
// (r.1 vanishes up to rounding: r stays orthogonal to the constant vector).
// The third L1 test needs |z|_1, which only every 10th iteration reads; on
// those iterations kb_yzr leaves the column's test, maxtime and maxits (in the
// reference's order) to kb_pupdate_z, which forms z while it updates p and
// sums |z|_1 on the way.  p of a column stopped by those tests is updated
// once more, which nothing reads: x comes from bestx.
template <typename T, bool kLoop = true>
__global__ void __launch_bounds__(kVecThreads) kb_yzr(int n, int kp, const T* __restrict__ y, const T* __restrict__ r,
                                                      PcgState* st, BatchShared* bs, double* partials, double eps,
                                                      LoopCtl ctl) {
  if (bs->all_done) return;
  using VT = Vec16<T>;
  constexpr int W = VT::W;
  using V = typename VT::V;
  const size_t NW = (size_t)n * kp / W;
  const size_t S = (size_t)gridDim.x * blockDim.x;
  size_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const V* yv4 = reinterpret_cast<const V*>(y);
  const V* rv4 = reinterpret_cast<const V*>(r);
  double acc[3][W];
#pragma unroll
  for (int j = 0; j < W; ++j) acc[0][j] = acc[1][j] = acc[2][j] = 0.0;
  for (; i + (kBU - 1) * S < NW; i += kBU * S) {
    V yv[kBU], rv[kBU];
#pragma unroll
    for (int u = 0; u < kBU; ++u) {
      yv[u] = yv4[i + u * S];
      rv[u] = rv4[i + u * S];
    }
#pragma unroll
    for (int u = 0; u < kBU; ++u) {
      T a[W], b[W];
      VT::split(yv[u], a);
      VT::split(rv[u], b);
#pragma unroll
      for (int j = 0; j < W; ++j) {
        acc[0][j] += (double)a[j];
        acc[1][j] += (double)a[j] * (double)b[j];
        acc[2][j] += (double)b[j];
      }
    }
  }
  for (; i < NW; i += S) {
    T a[W], b[W];
    VT::split(yv4[i], a);
    VT::split(rv4[i], b);
#pragma unroll
    for (int j = 0; j < W; ++j) {
      acc[0][j] += (double)a[j];
      acc[1][j] += (double)a[j] * (double)b[j];
      acc[2][j] += (double)b[j];
    }
  }
  double tot[3];
  if (batch_reduce_v<3, W>(acc, kp, partials, bs, 8, tot)) {
    const int c = threadIdx.x;
    bool deferred = false;
    if (c < kp) {
      const double mu = tot[0] / (double)n;
      st[c].mean = mu;
      if (bs->sweep_error && !st[c].done) mark_stop(&st[c], kSweepTimeout);
      if (!st[c].done && st[c].entering) {
        pcg_scalar_enter(&st[c], tot[1] - mu * tot[2]);
      } else if (!st[c].done && !pcg_scalar_rho(&st[c], tot[1] - mu * tot[2])) {
        if (st[c].itcnt % 10 == 0)
          deferred = true;
        else
          pcg_scalar_tail(&st[c], eps);
      }
    }
    const int any = __syncthreads_or(deferred);
    if (threadIdx.x == 0) bs->l1_due = any;
    batch_check_all<kLoop>(st, bs, kp, ctl);
  }
}

// z = y - mean, p = z + beta p (columns still running); on the iterations
// kb_yzr deferred, also |z|_1 and the deferred tests.  A vector whose columns
// have all stopped is skipped.
template <typename T, bool kLoop = true>
__global__ void __launch_bounds__(kVecThreads) kb_pupdate_z(int n, int kp, const T* __restrict__ y, T* __restrict__ p,
                                                            PcgState* st, BatchShared* bs, double* partials,
                                                            double eps, LoopCtl ctl) {
  if (bs->all_done) return;
  const bool l1 = bs->l1_due != 0;  // the same for every thread of the launch
  using VT = Vec16<T>;
  constexpr int W = VT::W;
  using V = typename VT::V;
  const size_t NW = (size_t)n * kp / W;
  const size_t S = (size_t)gridDim.x * blockDim.x;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c0 = (int)((i0 * W) % kp);
  double mu[W], beta[W];
  bool any = false;
#pragma unroll
  for (int j = 0; j < W; ++j) {
    mu[j] = st[c0 + j].mean;
    beta[j] = st[c0 + j].beta;
    any |= !st[c0 + j].done;
  }
  const V* yv4 = reinterpret_cast<const V*>(y);
  V* pv4 = reinterpret_cast<V*>(p);
  double acc[1][W];
#pragma unroll
  for (int j = 0; j < W; ++j) acc[0][j] = 0.0;
  size_t i = any ? i0 : NW;
  for (; i + (kBU - 1) * S < NW; i += kBU * S) {
    V yv[kBU], pv[kBU];
#pragma unroll
    for (int u = 0; u < kBU; ++u) {
      yv[u] = yv4[i + u * S];
      pv[u] = pv4[i + u * S];
    }
#pragma unroll
    for (int u = 0; u < kBU; ++u) {
      T a[W], b[W], o[W];
      VT::split(yv[u], a);
      VT::split(pv[u], b);
#pragma unroll
      for (int j = 0; j < W; ++j) {
        const T z = (T)((double)a[j] - mu[j]);
        o[j] = (T)((double)z + beta[j] * (double)b[j]);
        acc[0][j] += fabs((double)z);
      }
      pv4[i + u * S] = VT::join(o);
    }
  }
  for (; i < NW; i += S) {
    T a[W], b[W], o[W];
    VT::split(yv4[i], a);
    VT::split(pv4[i], b);
#pragma unroll
    for (int j = 0; j < W; ++j) {
      const T z = (T)((double)a[j] - mu[j]);
      o[j] = (T)((double)z + beta[j] * (double)b[j]);
      acc[0][j] += fabs((double)z);
    }
    pv4[i] = VT::join(o);
  }
  if (!l1) return;
  double tot[1];
  if (batch_reduce_v<1, W>(acc, kp, partials, bs, 9, tot)) {
    const int cc = threadIdx.x;
    if (cc < kp && !st[cc].done && st[cc].itcnt > 0 && st[cc].itcnt % 10 == 0) {
      st[cc].sum_abs_z = tot[0];
      pcg_scalar_tail(&st[cc], eps);
    }
    batch_check_all<kLoop>(st, bs, kp, ctl);
  }
}

// Timing only (acg_time_kernels_batch): every column running, mid-solve, with
// scalars that no stop test fires on (itcnt 1, tol 0, no maxits, no maxtime),
// so each timed vector kernel does its full pass.
__global__ void kb_timing_state(PcgState* st, BatchShared* bs, int kp) {
  const int c = threadIdx.x;
  if (c < kp) {
    PcgState* s = &st[c];
    s->tol = 0.0;
    s->maxtime_s = 1e300;
    s->maxits = 1ll << 62;
    s->stag_test = 0;
    s->nb = 1.0;
    s->rho = s->best_rho = 1.0;
    s->bestnr = 1.0;
    s->itcnt = 1;
    s->stag_count = 0;
    s->done = 0;
    s->xcur = 0;
    s->xnext = 1;
    s->xbest = 0;
  }
  if (c == 0) {
    bs->all_done = 0;
    bs->l1_due = 0;
    bs->pq_full = 1;  // kb_pq times its full pass (the every-10th steps)
  }
}

// ---- set-up and wrap-up ------------------------------------------------------

// External right-hand-side blocks (column c of B contiguous in the caller's
// vertex order) and the internal vertex-major rows (kp values per vertex, in
// level order) are transposes of each other through the vertex permutation.
// The gather and the scatter go through a shared-memory tile of kTrV external
// vertices: each column's kTrV values move as one contiguous 256-byte run and
// each vertex's kp values as one contiguous row, so both sides are coalesced
// (element-wise, consecutive threads touched kp different columns: 1.45 and
// 2.51 ms for 64 columns on the 1M grid).
constexpr int kTrV = 32;

// bint[iperm[e]*kp + c] = B[c*ldb + e] for c < k, 0 for padding; per-column mean.
__global__ void __launch_bounds__(kVecThreads) kb_gather_in(int n, int kp, const int* __restrict__ iperm,
                                                            const double* __restrict__ B, long long ldb,
                                                            double* __restrict__ bint, PcgState* st, BatchShared* bs,
                                                            double* partials) {
  __shared__ double tile[kTrV][kMaxBatch + 1];
  const int k = bs->k;
  const int t = threadIdx.x;
  const int per = (int)blockDim.x / kp, part = t / kp, col = t % kp;
  double acc[1] = {0.0};
  const int ntiles = (n + kTrV - 1) / kTrV;
  for (int tb = blockIdx.x; tb < ntiles; tb += gridDim.x) {
    const int e0 = tb * kTrV;
    for (int q = t; q < kTrV * kp; q += blockDim.x) {
      const int c = q / kTrV, e = q % kTrV;
      tile[e][c] = (c < k && e0 + e < n) ? B[(size_t)c * ldb + e0 + e] : 0.0;
    }
    __syncthreads();
    // column sums in a fixed order: thread t sums column t % kp over its rows
    for (int e = part; e < kTrV; e += per) acc[0] += tile[e][col];
    for (int q = t; q < kTrV * kp; q += blockDim.x) {
      const int e = q / kp, c = q % kp;
      if (e0 + e < n) bint[(size_t)iperm[e0 + e] * kp + c] = tile[e][c];
    }
    __syncthreads();
  }
  double tot[1];
  if (batch_reduce<1>(acc, kp, partials, &bs->counter[4], tot)) {
    const int c = threadIdx.x;
    if (c < kp) st[c].mean = tot[0] / (double)n;
  }
}

// bm = b - mean; r = bm (as T); x0 = 0; s, y pending; per-column |b| and reset.
template <typename T>
__global__ void __launch_bounds__(kVecThreads) kb_center(int n, int kp, double* __restrict__ bm, T* __restrict__ r,
                                                         T* __restrict__ x0, T* __restrict__ s_out, T* __restrict__ y_out,
                                                         PcgState* st, BatchShared* bs, double* partials, LoopCtl ctl) {
  const size_t N = (size_t)n * kp;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  const double mu = st[c].mean;
  const T pend = pending_value<T>();
  double acc[2] = {0.0, 0.0};
  for (size_t i = i0; i < N; i += (size_t)gridDim.x * blockDim.x) {
    const double v = bm[i] - mu;
    bm[i] = v;
    r[i] = (T)v;
    x0[i] = T(0);
    if (s_out) s_out[i] = pend;
    if (y_out) y_out[i] = pend;
    acc[0] += v * v;
    acc[1] += fabs(v);
  }
  double tot[2];
  if (batch_reduce<2>(acc, kp, partials, &bs->counter[5], tot)) {
    const int cc = threadIdx.x;
    if (cc < kp) {
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
      s->t_start = globaltimer_ns();
      if (s->nb == 0.0) {
        s->nr_true = 0.0;
        s->nr = 0.0;
        s->outer_done = 1;
        mark_stop(s, kConverged);
      } else if (!isfinite(s->nb)) {  // a NaN or Inf entry in this column
        s->outer_done = 1;
        mark_stop(s, kBadInput);
      }
    }
    if (threadIdx.x == 0) {
      bs->sweep_error = 0;
      bs->all_done = 0;
    }
    batch_check_all(st, bs, kp, ctl);
  }
}

template <typename T>
__global__ void __launch_bounds__(kVecThreads) kb_take_best(int n, int kp, const T* __restrict__ x3,
                                                            double* __restrict__ xf, const PcgState* st) {
  const size_t N = (size_t)n * kp;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  const T* xb = x3 + (size_t)st[c].xbest * N;
  for (size_t i = i0; i < N; i += (size_t)gridDim.x * blockDim.x) xf[i] = (double)xb[i];
}

// t = bm - L x (FP64), optionally stored; per column |t| -> nr_true, scale.
// Rows as kb_spmv walks them: 8 entries at a time shared inside the group of 8
// lanes, every gathered row of x issued before the first multiply-add (one
// entry at a time it took 1.10 ms for 64 columns on the 1M grid); the
// per-column sums of t^2 in two levels (batch_reduce_v).
template <int CPL>
__global__ void __launch_bounds__(kVecThreads) kb_true_residual(int n, const int* __restrict__ ptr,
                                                                const int* __restrict__ idx,
                                                                const double* __restrict__ val,
                                                                const double* __restrict__ x,
                                                                const double* __restrict__ bm, double* __restrict__ rout,
                                                                PcgState* st, BatchShared* bs, double* partials,
                                                                const int* gate = nullptr) {
  if (gate && !*gate) return;  // serving loop: only on ticks where some column needs it
  constexpr int kp = CPL * kBatchLanes;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int gl = gt & 7;
  const unsigned gmask = 0xffu << (threadIdx.x & 24);  // this group's lanes
  const int groups = gridDim.x * blockDim.x / 8;
  double sq[1][CPL];
#pragma unroll
  for (int j = 0; j < CPL; ++j) sq[0][j] = 0.0;
  int row = gt / 8;
  int n0 = row < n ? __ldg(&ptr[row]) : 0, n1 = row < n ? __ldg(&ptr[row + 1]) : 0;
  for (; row < n; row += groups) {
    const int k0 = n0, k1 = n1;
    const int nxt = row + groups;
    n0 = nxt < n ? __ldg(&ptr[nxt]) : 0;
    n1 = nxt < n ? __ldg(&ptr[nxt + 1]) : 0;
    double acc[CPL];
#pragma unroll
    for (int j = 0; j < CPL; ++j) acc[j] = 0.0;
    for (int kb = k0; kb < k1; kb += 8) {
      const int k = kb + gl;
      const int myid = k < k1 ? __ldg(&idx[k]) : -1;
      const double myc = k < k1 ? __ldg(&val[k]) : 0.0;
      int ids[8];
      double cs[8];
      double v[8][CPL];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        ids[u] = __shfl_sync(gmask, myid, u, 8);
        cs[u] = __shfl_sync(gmask, myc, u, 8);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (ids[u] >= 0) ldg_row<double, CPL>(v[u], x + (size_t)ids[u] * kp + gl * CPL);
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (ids[u] >= 0) {
#pragma unroll
          for (int j = 0; j < CPL; ++j) acc[j] += cs[u] * v[u][j];
        }
    }
    double b[CPL];
    ldg_row<double, CPL>(b, bm + (size_t)row * kp + gl * CPL);
#pragma unroll
    for (int j = 0; j < CPL; ++j) {
      const double t = b[j] - acc[j];
      if (rout) rout[(size_t)row * kp + gl * CPL + j] = t;
      sq[0][j] += t * t;
    }
  }
  double tot[1];
  if (batch_reduce_v<1, CPL>(sq, kp, partials, bs, 6, tot)) {
    const int c = threadIdx.x;
    if (c < kp) {
      PcgState* p = &st[c];
      p->scale = sqrt(tot[0]);
      p->nr_true = p->nb64 > 0.0 ? p->scale / p->nb64 : 0.0;
    }
  }
}

// X[c*ldx + e] = xf[iperm[e]*kp + c], c < k (the transpose of kb_gather_in).
__global__ void __launch_bounds__(kVecThreads) kb_scatter_out(int n, int kp, const int* __restrict__ iperm,
                                                              const double* __restrict__ xf, double* __restrict__ X,
                                                              long long ldx, const BatchShared* bs) {
  __shared__ double tile[kTrV][kMaxBatch + 1];
  const int k = bs->k;
  const int t = threadIdx.x;
  const int ntiles = (n + kTrV - 1) / kTrV;
  for (int tb = blockIdx.x; tb < ntiles; tb += gridDim.x) {
    const int e0 = tb * kTrV;
    for (int q = t; q < kTrV * kp; q += blockDim.x) {
      const int e = q / kp, c = q % kp;
      tile[e][c] = e0 + e < n ? xf[(size_t)iperm[e0 + e] * kp + c] : 0.0;
    }
    __syncthreads();
    for (int q = t; q < kTrV * kp; q += blockDim.x) {
      const int c = q / kTrV, e = q % kTrV;
      if (c < k && e0 + e < n) X[(size_t)c * ldx + e0 + e] = tile[e][c];
    }
    __syncthreads();
  }
}

// ---- mixed precision outer loop (per column) ---------------------------------

template <typename T>
__global__ void __launch_bounds__(kVecThreads) kb_outer_prep(int n, int kp, const double* __restrict__ r64,
                                                             T* __restrict__ rin, T* __restrict__ x0,
                                                             T* __restrict__ s_out, T* __restrict__ y_out, PcgState* st,
                                                             BatchShared* bs, double* partials, LoopCtl inner_ctl) {
  const size_t N = (size_t)n * kp;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  const bool act = !st[c].outer_done;
  const double inv = act ? 1.0 / st[c].scale : 0.0;
  const T pend = pending_value<T>();
  double acc[2] = {0.0, 0.0};
  for (size_t i = i0; i < N; i += (size_t)gridDim.x * blockDim.x) {
    const T v = act ? (T)(r64[i] * inv) : T(0);
    rin[i] = v;
    x0[i] = T(0);
    s_out[i] = pend;
    y_out[i] = pend;
    acc[0] += (double)v * (double)v;
    acc[1] += fabs((double)v);
  }
  double tot[2];
  if (batch_reduce<2>(acc, kp, partials, &bs->counter[7], tot)) {
    const int cc = threadIdx.x;
    if (cc < kp) {
      PcgState* s = &st[cc];
      if (s->outer_done) {
        s->done = 1;
      } else {
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
        if (s->nb == 0.0) mark_stop(s, kConverged);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      bool all = true;
      for (int q = 0; q < kp; ++q) all &= (st[q].done != 0);
      bs->all_done = all ? 1 : 0;
      if (inner_ctl.use_handle) cudaGraphSetConditional(inner_ctl.handle, all ? 0u : 1u);
    }
  }
}

// x64 += scale * x_in[best] for columns still refining
template <typename T>
__global__ void __launch_bounds__(kVecThreads) kb_outer_correct(int n, int kp, const T* __restrict__ x3,
                                                                double* __restrict__ x64, const PcgState* st) {
  const size_t N = (size_t)n * kp;
  const size_t i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(i0 % kp);
  if (st[c].outer_done) return;
  const T* xb = x3 + (size_t)st[c].xbest * N;
  const double sc = st[c].scale;
  for (size_t i = i0; i < N; i += (size_t)gridDim.x * blockDim.x) x64[i] += sc * (double)xb[i];
}

// per column: account iterations, decide, set the next inner tolerance
__global__ void kb_outer_decide(PcgState* st, BatchShared* bs, int kp, LoopCtl outer_ctl) {
  const int c = threadIdx.x;
  if (c < kp) {
    PcgState* s = &st[c];
    if (!s->outer_done) {
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
      } else {
        double it = 0.5 * s->tol_user / s->nr_true;
        if (it < s->min_inner_tol) it = s->min_inner_tol;
        if (it > 0.25) it = 0.25;
        s->inner_tol = it;
        s->maxits = s->maxits_user - s->total_its;
      }
    }
  }
  __syncthreads();
  if (c == 0) {
    bool all = true;
    for (int q = 0; q < kp; ++q) all &= (st[q].outer_done != 0);
    if (all && outer_ctl.use_handle) cudaGraphSetConditional(outer_ctl.handle, 0u);
  }
}

}  // namespace acg
