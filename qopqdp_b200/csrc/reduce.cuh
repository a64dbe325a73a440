// reduce.cuh -- deterministic FP64 grid reductions.
//
// Every block folds its threads with warp shuffles and a shared-memory
// tree, writes one partial per block, and the last block to finish (atomic
// ticket) sums the partials in a fixed order and publishes the result in
// device memory.  For a fixed grid the summation order never changes, so
// results are bit-reproducible run to run, and the completion ticket is
// reset by the last block so the next reduction needs no memset.
// Accumulation is always in double, for FP64, FP32 and FP16 fields alike.
#pragma once
#include "qopb.h"

namespace qopb {

constexpr int RED_THREADS = 256;

template <int N>
__device__ inline void warp_sum(double (&v)[N]) {
#pragma unroll
  for (int k = 0; k < N; k++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
}

// block-wide sum; result valid in thread 0 only
template <int N>
__device__ inline void block_sum(double (&v)[N]) {
  __shared__ double sh[32 * N];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  warp_sum<N>(v);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < N; k++) sh[w * N + k] = v[k];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < N; k++) v[k] = lane < nw ? sh[lane * N + k] : 0.0;
    warp_sum<N>(v);
  }
}

// called by every thread of every block with its private accumulators;
// the last block writes the grid total to res[0..N-1] and returns true in
// thread 0 so that a caller may run a scalar epilogue there.  `bid` / `nb`
// name the block within the set of blocks that reduce together (several
// independent reductions may share one launch, each with its own partials
// and ticket).
template <int N>
__device__ inline bool group_sum(double (&v)[N], double *part, unsigned *count, double *res, int bid, int nb) {
  block_sum<N>(v);
  __shared__ bool am_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < N; k++) part[bid * N + k] = v[k];
    __threadfence();
    unsigned t = atomicAdd(count, 1u);
    am_last = (t == (unsigned)nb - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  double s[N];
#pragma unroll
  for (int k = 0; k < N; k++) s[k] = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < N; k++) s[k] += __ldcg(part + b * N + k);
  block_sum<N>(s);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < N; k++) res[k] = s[k];
    *count = 0u;
    return true;
  }
  return false;
}

template <int N>
__device__ inline bool grid_sum(double (&v)[N], double *part, unsigned *count, double *res) {
  return group_sum<N>(v, part, count, res, blockIdx.x, gridDim.x);
}

// grid size for reductions: fixed per element count so the order is fixed
inline int red_grid(i64 n) {
  i64 b = (n + RED_THREADS - 1) / RED_THREADS;
  int cap = ctx().red_blocks;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

template <int N, class F>
__global__ void __launch_bounds__(RED_THREADS) k_reduce(F f, i64 n, double *part, unsigned *count, double *res) {
  double acc[N];
#pragma unroll
  for (int k = 0; k < N; k++) acc[k] = 0.0;
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) f(i, acc);
  grid_sum<N>(acc, part, count, res);
}

// launches the reduction and returns the N sums to the host (synchronous)
template <int N, class F>
void run_reduce(const F &f, i64 n, double *out) {
  Context &c = ctx();
  k_reduce<N, F><<<red_grid(n), RED_THREADS, 0, c.s>>>(f, n, c.d_part, c.d_count, c.d_res);
  QLAUNCH();
  dd_allreduce(c.d_res, N);
  QCHECK(cudaMemcpyAsync(c.h_res, c.d_res, sizeof(double) * N, cudaMemcpyDeviceToHost, c.s));
  QCHECK(cudaStreamSynchronize(c.s));
  for (int k = 0; k < N; k++) out[k] = c.h_res[k];
}

template <class F>
__global__ void k_map(F f, i64 n) {
  for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) f(i);
}

template <class F>
void run_map(const F &f, i64 n) {
  if (n <= 0) return;
  int grid = grid_for(n, 256);
  int cap = ctx().red_blocks * 4;
  if (grid > cap) grid = cap;
  k_map<F><<<grid, 256, 0, ctx().s>>>(f, n);
  QLAUNCH();
}

}  // namespace qopb
