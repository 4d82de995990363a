// msg_common.cuh -- shared helpers for the B200 Newton-Krylov library.
//
// Every translation unit is compiled with --fmad=false so that products and sums
// round separately, in the order the Fortran reference evaluates them; the
// helpers below keep that explicit where it matters.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

namespace msg {

// ---------------------------------------------------------------------------------
// Error handling: no exception crosses the C ABI.  Host helpers record the first
// CUDA error in a thread-local message and return a status code.
// ---------------------------------------------------------------------------------
void set_error(const char *fmt, ...);
const char *get_error();

#define MSG_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      ::msg::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
      return MSG_ERR_CUDA;                                                              \
    }                                                                                   \
  } while (0)

extern long long g_launches;   // kernels launched by this library (all contexts)

#define MSG_CHECK_LAUNCH()                                                              \
  do {                                                                                  \
    __atomic_fetch_add(&::msg::g_launches, 1LL, __ATOMIC_RELAXED);                      \
    cudaError_t e_ = cudaGetLastError();                                                \
    if (e_ != cudaSuccess) {                                                            \
      ::msg::set_error("%s:%d launch: %s", __FILE__, __LINE__, cudaGetErrorString(e_)); \
      return MSG_ERR_CUDA;                                                              \
    }                                                                                   \
  } while (0)

constexpr int kNumSM = 148;          // B200
constexpr int kRedBlocks = 4 * kNumSM;   // fixed grid for deterministic two-stage reductions
constexpr int kThreads = 256;

// Face directions (reference conn_dir - 1): up, north, west, east, south, down.
enum Dir { UP = 0, NORTH = 1, WEST = 2, EAST = 3, SOUTH = 4, DOWN = 5 };

// Upstream selection (Calc_parameter.f90:107-125): kr of cell i when h_i >= h_j.
__device__ __forceinline__ double upwind(double head_dif, double c1, double c2) {
  return head_dif >= 0.0 ? c1 : c2;
}

// Block-wide sum of one double (deterministic for a fixed block size).
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(0xffffffffu, v, o));
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NT / 32; ++i) r = __dadd_rn(r, sh[i]);
  }
  __syncthreads();
  return r;   // valid in thread 0
}

// Sum a partials array of fixed length in index order (one thread).
__device__ __forceinline__ double sum_partials(const double *p, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = __dadd_rn(s, p[i]);
  return s;
}

}  // namespace msg
