// Dense tail of the LDLinv sweeps.
//
// The final levels of the LDLinv dependency DAG hold few vertices but most of
// its depth (on a 1M-vertex 3D grid the last 4096 vertices span 513 of 977
// levels): the approximate elimination ends in a nearly dense Schur
// complement.  The vertices of levels >= L0 form a set T closed under
// successors, so with the unit lower-triangular forward operator (I - C)
// split into head H and tail T blocks,
//
//   forward   s_T = M (r_T + C_TH s_H),          M = (I - C_TT)^{-1}
//   backward  y_T = M^T (g_T * s_T),              y_H from the usual sweep
//
// which is the operator of src/approxChol.jl:1347-1408 restricted to T, with
// the substitution over T's levels replaced by one dense triangular product
// (M is computed once, in FP64, when the solver is built).  The sweep writes
// w_T = r_T + C_TH s_H for the tail vertices (their tail inputs are left out
// of the sweep's entry lists); the kernels below form s_T = M w_T and
// y_T = M^T (g_T s_T).
//
// Layout: M is K x K row-major (K = |T|, rows and columns in internal vertex
// order, which is topological inside T, so M is lower triangular).  Vectors
// are vertex-major with kp values per vertex (kp = 1 for one right-hand side).
// A product is split over CTAs by (row tile of kDenseRows outputs, chunk of
// kDenseChunk reduction indices); each CTA writes a partial tile and
// kd_reduce sums the chunks of a row in chunk order, so results do not depend
// on scheduling.
#pragma once

#include "acg_kernels.cuh"

namespace acg {

constexpr int kDenseRows = 64;
constexpr int kDenseChunk = 256;
constexpr int kDenseSub = 64;
constexpr int kDenseThreads = 256;
constexpr int kDenseDefaultK = 4096;  // largest tail chosen automatically
constexpr int kDenseMaxK = 8192;      // largest tail accepted
constexpr int kDenseMinLevels = 8;    // fewer tail levels than this: no dense tail

__host__ __device__ constexpr int dense_chunks(int K) { return (K + kDenseChunk - 1) / kDenseChunk; }
__host__ __device__ constexpr int dense_row_tiles(int K) { return (K + kDenseRows - 1) / kDenseRows; }

// Does reduction chunk kc meet row tile rt inside the triangle?  Forward
// (M, lower): columns j <= i; backward (M^T, upper): rows j >= i.
__host__ __device__ __forceinline__ bool dense_active(bool fwd, int rt, int kc) {
  return fwd ? (kc * kDenseChunk <= rt * kDenseRows + kDenseRows - 1)
             : (kc * kDenseChunk + kDenseChunk - 1 >= rt * kDenseRows);
}

// part[kc][i][c] = sum over j in chunk kc (inside the triangle) of A[i][j] * src[j][c],
// A = M (forward) or M^T (backward, src scaled by g); kp = 8 * CPL columns.
// Register tiling: the 256 threads form RG row groups x CG column groups and
// each computes RT rows x CT columns of the 64-row tile, so one stage of SUB
// reduction indices costs RT + CT shared-memory loads per RT * CT FMAs.
template <typename T, int CPL, bool kFwd>
__global__ void __launch_bounds__(kDenseThreads) kd_partial(int K, const T* __restrict__ M, const T* __restrict__ src,
                                                            const T* __restrict__ g, T* __restrict__ part,
                                                            const int* __restrict__ done) {
  if (done && *done) return;
  const int rt = blockIdx.x, kc = blockIdx.y;
  if (!dense_active(kFwd, rt, kc)) return;
  constexpr int kp = 8 * CPL;
  constexpr int CT = kp >= 32 ? kp / 16 : 1;       // columns per thread
  constexpr int CG = kp / CT;                      // column groups
  constexpr int RG = kDenseThreads / CG;           // row groups
  constexpr int RT = kDenseRows / RG;              // rows per thread
  constexpr int SUB = 32;                          // reduction indices per stage
  static_assert(CG * RG == kDenseThreads && RT * RG == kDenseRows, "dense tile shape");
  __shared__ T As[kDenseRows][SUB + 1];            // A tile, row-major, padded
  __shared__ __align__(16) T Bs[SUB][kp];
  const int tid = threadIdx.x;
  const int rg = tid / CG, cg = tid % CG;
  const int i0 = rt * kDenseRows;
  T acc[RT][CT];
#pragma unroll
  for (int a = 0; a < RT; ++a)
#pragma unroll
    for (int b = 0; b < CT; ++b) acc[a][b] = T(0);
  const int jend = min(K, kc * kDenseChunk + kDenseChunk);
  for (int j0 = kc * kDenseChunk; j0 < jend; j0 += SUB) {
    for (int e = tid; e < kDenseRows * SUB; e += kDenseThreads) {
      // forward reads rows of M along j, backward reads rows of M along i:
      // both coalesced, both conflict-free in shared memory
      const int rr = kFwd ? e / SUB : e % kDenseRows;
      const int jj = kFwd ? e % SUB : e / kDenseRows;
      const int ii = i0 + rr, j = j0 + jj;
      T a = T(0);
      if (ii < K && j < K && (kFwd ? j <= ii : j >= ii)) a = kFwd ? M[(size_t)ii * K + j] : M[(size_t)j * K + ii];
      As[rr][jj] = a;
    }
    for (int e = tid; e < SUB * kp; e += kDenseThreads) {
      const int jj = e / kp, c = e % kp, j = j0 + jj;
      T b = T(0);
      if (j < K) {
        b = src[(size_t)j * kp + c];
        if (!kFwd) b *= g[j];
      }
      Bs[jj][c] = b;
    }
    __syncthreads();
#pragma unroll 4
    for (int jj = 0; jj < SUB; ++jj) {
      T a[RT], b[CT];
#pragma unroll
      for (int q = 0; q < RT; ++q) a[q] = As[rg * RT + q][jj];
#pragma unroll
      for (int q = 0; q < CT; ++q) b[q] = Bs[jj][cg * CT + q];
#pragma unroll
      for (int x = 0; x < RT; ++x)
#pragma unroll
        for (int y = 0; y < CT; ++y) acc[x][y] += a[x] * b[y];
    }
    __syncthreads();
  }
#pragma unroll
  for (int x = 0; x < RT; ++x) {
    const int i = i0 + rg * RT + x;
    if (i < K) {
#pragma unroll
      for (int y = 0; y < CT; ++y) part[((size_t)kc * K + i) * kp + cg * CT + y] = acc[x][y];
    }
  }
}

// One right-hand side: the same partial products with a warp per output row
// (forward, coalesced along a row of M) or a lane per output row (backward,
// coalesced along a row of M = a column of M^T).
template <typename T, bool kFwd>
__global__ void __launch_bounds__(kDenseThreads) kd1_partial(int K, const T* __restrict__ M, const T* __restrict__ src,
                                                             const T* __restrict__ g, T* __restrict__ part,
                                                             const int* __restrict__ done, int vs) {
  if (done && *done) return;
  const int rt = blockIdx.x, kc = blockIdx.y;
  if (!dense_active(kFwd, rt, kc)) return;
  __shared__ T Bs[kDenseChunk];
  __shared__ T red[kDenseThreads / 32][33];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int i0 = rt * kDenseRows, j0 = kc * kDenseChunk;
  for (int jj = tid; jj < kDenseChunk; jj += kDenseThreads) {
    const int j = j0 + jj;
    T b = T(0);
    if (j < K) {
      b = src[(size_t)j * vs];
      if (!kFwd) b *= g[j];
    }
    Bs[jj] = b;
  }
  __syncthreads();
  if (kFwd) {
    for (int rr = w; rr < kDenseRows; rr += kDenseThreads / 32) {
      const int i = i0 + rr;
      T acc = T(0);
      if (i < K) {
        for (int jj = lane; jj < kDenseChunk; jj += 32) {
          const int j = j0 + jj;
          if (j <= i && j < K) acc += M[(size_t)i * K + j] * Bs[jj];
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0 && i < K) part[(size_t)kc * K + i] = acc;
    }
  } else {
    for (int h = 0; h < kDenseRows / 32; ++h) {
      const int i = i0 + h * 32 + lane;
      T acc = T(0);
      if (i < K) {
        for (int jj = w * 32; jj < w * 32 + 32; ++jj) {
          const int j = j0 + jj;
          if (j >= i && j < K) acc += M[(size_t)j * K + i] * Bs[jj];
        }
      }
      red[w][lane] = acc;
      __syncthreads();
      if (w == 0) {
        T sum = T(0);
#pragma unroll
        for (int q = 0; q < kDenseThreads / 32; ++q) sum += red[q][lane];
        if (i < K) part[(size_t)kc * K + i] = sum;
      }
      __syncthreads();
    }
  }
}

// dst[i * rs + c] = sum of the partial tiles of row i over its chunks, in chunk
// order (rs: the destination's row stride, kp for batched rows).
template <typename T, bool kFwd>
__global__ void __launch_bounds__(kVecThreads) kd_reduce(int K, int kp, const T* __restrict__ part, T* __restrict__ dst,
                                                         const int* __restrict__ done, int rs) {
  if (done && *done) return;
  const int nch = dense_chunks(K);
  const size_t N = (size_t)K * kp;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (size_t)gridDim.x * blockDim.x) {
    const int rt = (int)(e / kp) / kDenseRows;
    T sum = T(0);
    for (int kc = 0; kc < nch; ++kc)
      if (dense_active(kFwd, rt, kc)) sum += part[(size_t)kc * N + e];
    dst[(e / kp) * rs + e % kp] = sum;
  }
}

}  // namespace acg
