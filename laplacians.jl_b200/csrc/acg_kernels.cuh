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

namespace acg {

constexpr int kMaxPartialBlocks = 2048;
constexpr int kVecBlocks = 148 * 4;   // grid of the streaming vector kernels
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
  int pad1;
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

// One row / vertex per VL-lane group.  All lanes of a warp stay converged in
// the shuffles because the row loop bound is uniform per warp (rows are
// assigned in warp-aligned strides and the loop runs while any lane of the
// warp has work).
template <typename T, int VL>
__device__ __forceinline__ T row_dot(const int* __restrict__ ptr, const int* __restrict__ idx,
                                     const T* __restrict__ val, const T* x, int row, bool active, int lane) {
  T acc = T(0);
  if (active) {
    const int k1 = __ldg(&ptr[row + 1]);
    for (int k = __ldg(&ptr[row]) + lane; k < k1; k += VL) acc += __ldg(&val[k]) * x[__ldg(&idx[k])];
  }
  return group_sum<VL>(acc);
}

// Forward sweep, one level: s[v] = r[v] + sum coef * s[src], v in [v0, v1).
template <typename T, int VL>
__global__ void __launch_bounds__(256) k_fwd_level(int v0, int v1, const int* __restrict__ fptr,
                                                   const int* __restrict__ fidx, const T* __restrict__ fc,
                                                   const T* __restrict__ r, T* s, const PcgState* st) {
  if (st && st->done) return;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = gt & (VL - 1);
  const int v = v0 + gt / VL;
  const int wv = v0 + (gt & ~31) / VL;  // first vertex of this warp
  if (wv >= v1) return;                  // whole warp out of range
  const bool active = v < v1;
  T acc = row_dot<T, VL>(fptr, fidx, fc, s, v, active, lane);
  if (active && lane == 0) s[v] = r[v] + acc;
}

// Backward sweep, one level (in place): y[v] = g[v]*y[v] + sum coef * y[dst].
template <typename T, int VL>
__global__ void __launch_bounds__(256) k_bwd_level(int v0, int v1, const int* __restrict__ bptr,
                                                   const int* __restrict__ bidx, const T* __restrict__ bc,
                                                   const T* __restrict__ g, T* y, const PcgState* st) {
  if (st && st->done) return;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = gt & (VL - 1);
  const int v = v0 + gt / VL;
  const int wv = v0 + (gt & ~31) / VL;
  if (wv >= v1) return;
  const bool active = v < v1;
  T acc = row_dot<T, VL>(bptr, bidx, bc, y, v, active, lane);
  if (active && lane == 0) y[v] = g[v] * y[v] + acc;
}

// A run of thin levels [l0, l1) in one CTA: a block barrier between levels.
constexpr int kThinThreads = 512;
constexpr int kMaxThinLevels = 4096;

template <typename T, int VL>
__global__ void __launch_bounds__(kThinThreads) k_fwd_thin(int l0, int l1, const int* __restrict__ lvl_off,
                                                           const int* __restrict__ fptr, const int* __restrict__ fidx,
                                                           const T* __restrict__ fc, const T* __restrict__ r, T* s,
                                                           const PcgState* st) {
  if (st && st->done) return;
  __shared__ int off[kMaxThinLevels + 1];
  for (int i = threadIdx.x; i <= l1 - l0; i += blockDim.x) off[i] = lvl_off[l0 + i];
  __syncthreads();
  const int lane = threadIdx.x & (VL - 1);
  const int grp = threadIdx.x / VL;
  constexpr int kGroups = kThinThreads / VL;
  for (int l = 0; l < l1 - l0; ++l) {
    const int v0 = off[l], v1 = off[l + 1];
    for (int base = v0; base < v1; base += kGroups) {
      const int v = base + grp;
      const bool active = v < v1;
      T acc = row_dot<T, VL>(fptr, fidx, fc, s, v, active, lane);
      if (active && lane == 0) s[v] = r[v] + acc;
    }
    __syncthreads();
  }
}

template <typename T, int VL>
__global__ void __launch_bounds__(kThinThreads) k_bwd_thin(int l0, int l1, const int* __restrict__ lvl_off,
                                                           const int* __restrict__ bptr, const int* __restrict__ bidx,
                                                           const T* __restrict__ bc, const T* __restrict__ g, T* y,
                                                           const PcgState* st) {
  if (st && st->done) return;
  // walks levels l1-1 down to l0
  __shared__ int off[kMaxThinLevels + 1];
  for (int i = threadIdx.x; i <= l1 - l0; i += blockDim.x) off[i] = lvl_off[l0 + i];
  __syncthreads();
  const int lane = threadIdx.x & (VL - 1);
  const int grp = threadIdx.x / VL;
  constexpr int kGroups = kThinThreads / VL;
  for (int l = l1 - l0 - 1; l >= 0; --l) {
    const int v0 = off[l], v1 = off[l + 1];
    for (int base = v0; base < v1; base += kGroups) {
      const int v = base + grp;
      const bool active = v < v1;
      T acc = row_dot<T, VL>(bptr, bidx, bc, y, v, active, lane);
      if (active && lane == 0) y[v] = g[v] * y[v] + acc;
    }
    __syncthreads();
  }
}

}  // namespace acg
