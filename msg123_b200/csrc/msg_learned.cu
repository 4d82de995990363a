// msg_learned.cu -- learned Newton initial guess: a 3D CNN that predicts the next
// head increment from the current state, trained on steps the GPU solver generates.
//
// Network: four 3x3x3 convolutions, 16 channels, GELU after the first three, BF16
// weights and activations, FP32 accumulation and FP32 master weights (AdamW).  Inputs
// (channels-last, 16 channels, 7 used): pressure head, last increment / s, ln Ks,
// alpha, n, top recharge flag, dt ratio.  The output o is added to the plain linear
// extrapolation:  h_{t+1} = h_t + r (h_t - h_{t-1}) + s o,  s = rms(h_t - h_{t-1}),
// r = dt_new / dt_old, so an untrained (zero) head gives the extrapolation back.
//
// Inference inside the time loop (learned_guess) runs the convolutions on the tcgen05
// tensor cores with TMA-staged halo tiles and TMEM accumulators (msg_conv_tc.cu).
// Training (forward with saved pre-activations, input and weight gradients) uses
// implicit GEMMs with mma.sync m16n8k16 (BF16 x BF16 -> FP32): a warp owns 16
// consecutive cells (the M dimension), the 16 output channels are two n8 tiles, and
// each of the 27 taps is one k16 step over the 16 input channels.  The input-gradient
// pass is the same kernel with the taps mirrored and the weights transposed; the weight
// gradient reduces dz^T a over cells with the same instruction.
#include "msg_ctx.cuh"
#include "msg_conv_tc.cuh"
#include <cuda_bf16.h>
#include <vector>
#include <mutex>
#include <cmath>
#include <algorithm>

namespace msg {

constexpr int kC = 16, kTaps = 27, kLayers = 4;
constexpr int kWl = kTaps * kC * kC;         // weights per layer (W[tap][co][ci])
constexpr int kPl = kWl + kC;                 // + bias
constexpr int kNParam = kLayers * kPl;

struct Grid3 {
  int nx, ny, nz, nxy, N;
};

struct Sample {
  Grid3 g;
  __nv_bfloat16 *x;   // features [N][16]
  float *y;           // target [N]
};

struct Net {
  float *w32 = nullptr;                // [kNParam] master weights
  __nv_bfloat16 *w16 = nullptr;        // [kLayers][kWl]  W[tap][co][ci]
  __nv_bfloat16 *wt16 = nullptr;       // [kLayers][kWl]  mirrored taps, transposed
  __nv_bfloat16 *wtc = nullptr;        // tensor-core operand layout (conv_pack_weights)
  ConvPlan *plan = nullptr;            // padded activations + TMA maps of the inference grid
  // One network may be attached to several contexts (e.g. ensemble members driven by
  // concurrent worker threads): the inference buffers are the network's, so each guess
  // holds this lock until its stream has finished with them.
  std::recursive_mutex mu;
  float *m = nullptr, *v = nullptr, *grad = nullptr;
  float *part = nullptr;               // weight-gradient partials
  int part_cap = 0;
  int step = 0;
  float dead = 0.1f;                   // deadband on the normalised correction
  // activations (sized for the largest grid seen)
  int cap = 0;
  __nv_bfloat16 *a[kLayers] = {nullptr, nullptr, nullptr, nullptr};   // a[0] = input features
  float *z[kLayers] = {nullptr, nullptr, nullptr, nullptr};           // pre-activations (z[3]: output)
  __nv_bfloat16 *dz = nullptr;         // gradient of the current layer's pre-activation [N][16]
  __nv_bfloat16 *dz2 = nullptr;
  float *loss_part = nullptr;
  double *hpin = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<Sample> data;
  // bounded sample store: with store_cap > 0, a sample collected when the store is full
  // replaces a uniformly drawn stored one with probability store_cap / seen (reservoir sampling), so the
  // store stays a uniform sample of every step collected so far
  int store_cap = 0;
  long long seen = 0;
  unsigned long long rs = 0x2545F4914F6CDD1Dull;
};

}  // namespace msg

struct msg_cnn {
  msg::Net net;
};

namespace msg {

// ---------------------------------------------------------------------------------
// tensor-core primitive
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void mma_bf16(float d[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0,
                                         unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ int nbr(const Grid3 &g, int cell, int tap) {
  if (cell >= g.N) return -1;
  int z = cell / g.nxy, rem = cell - z * g.nxy, y = rem / g.nx, x = rem - y * g.nx;
  int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
  x += dx; y += dy; z += dz;
  if (x < 0 || x >= g.nx || y < 0 || y >= g.ny || z < 0 || z >= g.nz) return -1;
  return x + g.nx * (y + g.ny * z);
}

__device__ __forceinline__ unsigned ld2(const __nv_bfloat16 *p, int cell, int ch) {
  if (cell < 0) return 0u;
  return *reinterpret_cast<const unsigned *>(p + (size_t)cell * kC + ch);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Convolution over all 27 taps.  MODE 0: forward hidden layer (z, GELU -> a_out);
// MODE 1: forward output layer (channel 0 -> out); MODE 2: input gradient
// (acc * gelu'(zprev) -> dz_out).  W is [tap][co][ci] (already mirrored/transposed for MODE 2).
template <int MODE>
__global__ void __launch_bounds__(256) k_conv(Grid3 g, const __nv_bfloat16 *__restrict__ in,
                                              const __nv_bfloat16 *__restrict__ W, const float *__restrict__ bias,
                                              float *z_out, __nv_bfloat16 *a_out, float *out,
                                              const float *__restrict__ zprev, __nv_bfloat16 *dz_out) {
  __shared__ __align__(16) __nv_bfloat16 sw[kWl];
  for (int k = threadIdx.x; k < kWl / 8; k += blockDim.x)
    reinterpret_cast<uint4 *>(sw)[k] = reinterpret_cast<const uint4 *>(W)[k];
  __syncthreads();
  const int lane = threadIdx.x & 31, gq = lane >> 2, tq = lane & 3;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int c0 = warp * 16;
  if (c0 >= g.N) return;
  const int ca = c0 + gq, cb = c0 + gq + 8;
  float d0[4] = {0.f, 0.f, 0.f, 0.f}, d1[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 3
  for (int tap = 0; tap < kTaps; ++tap) {
    int na = nbr(g, ca, tap), nb2 = nbr(g, cb, tap);
    unsigned a0 = ld2(in, na, 2 * tq), a1 = ld2(in, nb2, 2 * tq);
    unsigned a2 = ld2(in, na, 2 * tq + 8), a3 = ld2(in, nb2, 2 * tq + 8);
    const __nv_bfloat16 *wt = sw + tap * kC * kC;
    unsigned b00 = *reinterpret_cast<const unsigned *>(wt + gq * kC + 2 * tq);
    unsigned b01 = *reinterpret_cast<const unsigned *>(wt + gq * kC + 2 * tq + 8);
    unsigned b10 = *reinterpret_cast<const unsigned *>(wt + (gq + 8) * kC + 2 * tq);
    unsigned b11 = *reinterpret_cast<const unsigned *>(wt + (gq + 8) * kC + 2 * tq + 8);
    mma_bf16(d0, a0, a1, a2, a3, b00, b01);
    mma_bf16(d1, a0, a1, a2, a3, b10, b11);
  }
  // epilogue: d0 -> channels 2t,2t+1 ; d1 -> 8+2t, 8+2t+1 ; [0,1] cell a, [2,3] cell b
  const int cells[2] = {ca, cb};
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int cell = cells[h];
    if (cell >= g.N) continue;
    float v[4] = {d0[2 * h], d0[2 * h + 1], d1[2 * h], d1[2 * h + 1]};
    int ch[4] = {2 * tq, 2 * tq + 1, 8 + 2 * tq, 9 + 2 * tq};
    if (MODE == 0) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        float zz = v[q] + bias[ch[q]];
        z_out[(size_t)cell * kC + ch[q]] = zz;
        a_out[(size_t)cell * kC + ch[q]] = __float2bfloat16(gelu(zz));
      }
    } else if (MODE == 1) {
      if (tq == 0) out[cell] = v[0] + bias[0];
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q)
        dz_out[(size_t)cell * kC + ch[q]] = __float2bfloat16(v[q] * gelu_d(zprev[(size_t)cell * kC + ch[q]]));
    }
  }
}

// Weight gradient: part[blk][tap][co][ci] = sum over this block's cells of
// dz[cell][co] * in[nbr(cell,tap)][ci]; bias gradient from tap 13 blocks (dz sums).
// grid = (chunks, 27); each warp walks 16-cell steps of the chunk.
constexpr int kWgChunk = 4096;
__global__ void __launch_bounds__(128) k_wgrad(Grid3 g, const __nv_bfloat16 *__restrict__ dz,
                                               const __nv_bfloat16 *__restrict__ in, float *part) {
  __shared__ float red[4][kC * kC];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, gq = lane >> 2, tq = lane & 3;
  const int tap = blockIdx.y;
  const int start = blockIdx.x * kWgChunk;
  float d0[4] = {0.f, 0.f, 0.f, 0.f}, d1[4] = {0.f, 0.f, 0.f, 0.f};
  for (int c0 = start + w * 16; c0 < min(start + kWgChunk, g.N); c0 += 64) {
    // A = dz^T (M = co, K = 16 cells): rows gq / gq+8, k = 2t,2t+1 / 2t+8,2t+9
    auto pk = [&](const __nv_bfloat16 *p, int cellA, int cellB, int ch) -> unsigned {
      unsigned lo = 0, hi = 0;
      if (cellA >= 0 && cellA < g.N) lo = __bfloat16_as_ushort(p[(size_t)cellA * kC + ch]);
      if (cellB >= 0 && cellB < g.N) hi = __bfloat16_as_ushort(p[(size_t)cellB * kC + ch]);
      return lo | (hi << 16);
    };
    int k0 = c0 + 2 * tq, k1 = c0 + 2 * tq + 1, k8 = c0 + 2 * tq + 8, k9 = c0 + 2 * tq + 9;
    unsigned a0 = pk(dz, k0, k1, gq), a1 = pk(dz, k0, k1, gq + 8);
    unsigned a2 = pk(dz, k8, k9, gq), a3 = pk(dz, k8, k9, gq + 8);
    // B = shifted input (K = cells, N = ci): n = gq (tile 0) / gq + 8 (tile 1)
    int n0 = (k0 < g.N) ? nbr(g, k0, tap) : -1, n1 = (k1 < g.N) ? nbr(g, k1, tap) : -1;
    int n8 = (k8 < g.N) ? nbr(g, k8, tap) : -1, n9 = (k9 < g.N) ? nbr(g, k9, tap) : -1;
    unsigned b00 = pk(in, n0, n1, gq), b01 = pk(in, n8, n9, gq);
    unsigned b10 = pk(in, n0, n1, gq + 8), b11 = pk(in, n8, n9, gq + 8);
    mma_bf16(d0, a0, a1, a2, a3, b00, b01);
    mma_bf16(d1, a0, a1, a2, a3, b10, b11);
  }
  // D[co][ci]: d0 -> (co gq / gq+8, ci 2t,2t+1), d1 -> ci + 8
  float *r = red[w];
  r[gq * kC + 2 * tq] = d0[0];       r[gq * kC + 2 * tq + 1] = d0[1];
  r[(gq + 8) * kC + 2 * tq] = d0[2]; r[(gq + 8) * kC + 2 * tq + 1] = d0[3];
  r[gq * kC + 8 + 2 * tq] = d1[0];       r[gq * kC + 9 + 2 * tq] = d1[1];
  r[(gq + 8) * kC + 8 + 2 * tq] = d1[2]; r[(gq + 8) * kC + 9 + 2 * tq] = d1[3];
  __syncthreads();
  for (int e = threadIdx.x; e < kC * kC; e += blockDim.x) {
    float s = red[0][e] + red[1][e] + red[2][e] + red[3][e];
    part[((size_t)blockIdx.x * kTaps + tap) * kC * kC + e] = s;
  }
}

// bias gradient partials: sum of dz over cells per channel
__global__ void __launch_bounds__(256) k_bgrad(Grid3 g, const __nv_bfloat16 *dz, float *part) {
  __shared__ float sh[256];
  int ch = threadIdx.x & 15;
  float s = 0.f;
  int start = blockIdx.x * kWgChunk;
  for (int c = start + (threadIdx.x >> 4); c < min(start + kWgChunk, g.N); c += 16)
    s += __bfloat162float(dz[(size_t)c * kC + ch]);
  sh[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < 16) {
    float t = 0.f;
    for (int k = 0; k < 16; ++k) t += sh[k * 16 + threadIdx.x];
    part[(size_t)blockIdx.x * kC + threadIdx.x] = t;
  }
}

// sum weight partials in chunk order into grad (deterministic)
__global__ void k_reduce_parts(int nchunks, const float *part, int len, float *grad) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= len) return;
  float s = 0.f;
  for (int k = 0; k < nchunks; ++k) s += part[(size_t)k * len + e];
  grad[e] = s;
}

// loss: dL/dout = 2 (out - y) / N, written as channel 0 of dz; partial sums of the squared error
__global__ void __launch_bounds__(256) k_loss(int n, const float *out, const float *y, __nv_bfloat16 *dz, double *part) {
  __shared__ double sh[8];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float e = out[i] - y[i];
    s += (double)e * e;
    __nv_bfloat16 *q = dz + (size_t)i * kC;
    q[0] = __float2bfloat16(2.0f * e / (float)n);
#pragma unroll
    for (int c = 1; c < kC; ++c) q[c] = __float2bfloat16(0.f);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += sh[w];
    part[blockIdx.x] = t;
  }
}

// AdamW on FP32 master weights, refresh the BF16 copies (forward and mirrored/transposed)
__global__ void k_adamw(int n, float *w, const float *gr, float *m, float *v, float lr, float b1, float b2, float eps,
                        float wd, float c1, float c2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = gr[i];
  float mi = b1 * m[i] + (1.f - b1) * gi;
  float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi; v[i] = vi;
  float mh = mi / c1, vh = vi / c2;
  w[i] = w[i] - lr * (mh / (sqrtf(vh) + eps) + wd * w[i]);
}

__global__ void k_pack_weights(const float *w32, __nv_bfloat16 *w16, __nv_bfloat16 *wt16) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kLayers * kWl) return;
  int l = e / kWl, r = e - l * kWl;
  int tap = r / (kC * kC), co = (r / kC) % kC, ci = r % kC;
  __nv_bfloat16 v = __float2bfloat16(w32[(size_t)l * kPl + r]);
  w16[e] = v;
  // input gradient: W'[26 - tap][ci][co] = W[tap][co][ci]
  wt16[(size_t)l * kWl + (size_t)(kTaps - 1 - tap) * kC * kC + ci * kC + co] = v;
}

// ---------------------------------------------------------------------------------
// features from the solver state (before the step): h_t = head_old, h_{t-1} = head_old2
// ---------------------------------------------------------------------------------
struct FeatArgs {
  Grid3 g;
  const double *h, *hprev, *top;
  const float *ksz, *reta, *retn;
  const double *calc_rech, *rech_base;
  double len_scal, inv_s, ratio;
};

// PAD = false: compact [N][16]; PAD = true: the padded chunk-planar layout of ConvPlan
// (plane = padded cells per chunk plane).
template <bool PAD>
__global__ void k_features(FeatArgs f, __nv_bfloat16 *x, long long plane) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f.g.N) return;
  float v[kC];
#pragma unroll
  for (int c = 0; c < kC; ++c) v[c] = 0.f;
  v[0] = (float)((f.h[i] - f.top[i]) * f.len_scal * 0.1);
  v[1] = (float)((f.h[i] - f.hprev[i]) * f.inv_s);
  v[2] = (logf((float)((double)f.ksz[i] * f.len_scal)) + 11.512925f) / 1.5f;
  v[3] = ((float)((double)f.reta[i] / f.len_scal) - 3.0f) / 1.5f;
  v[4] = (f.retn[i] - 1.9f) / 0.4f;
  if (i < f.g.nxy) v[5] = (f.rech_base[i] != 0.0) ? (float)(f.calc_rech[i] / f.rech_base[i]) : 0.f;
  v[6] = (float)f.ratio;
  __align__(16) __nv_bfloat16 q[kC];
#pragma unroll
  for (int c = 0; c < kC; ++c) q[c] = __float2bfloat16(v[c]);
  uint4 *dst = reinterpret_cast<uint4 *>(x);
  if (PAD) {
    int iz = i / f.g.nxy, rem = i - iz * f.g.nxy, iy = rem / f.g.nx, ix = rem - iy * f.g.nx;
    long long p = ((long long)(iz + 1) * (f.g.ny + 2) + (iy + 1)) * (f.g.nx + 2) + (ix + 1);
    dst[p] = reinterpret_cast<const uint4 *>(q)[0];
    dst[plane + p] = reinterpret_cast<const uint4 *>(q)[1];
  } else {
    dst[2 * (size_t)i] = reinterpret_cast<const uint4 *>(q)[0];
    dst[2 * (size_t)i + 1] = reinterpret_cast<const uint4 *>(q)[1];
  }
}

// target: ((h_{t+1} - h_t) - r (h_t - h_{t-1})) / s
__global__ void k_target(int n, const double *hn, const double *h, const double *hp, double ratio, double inv_s,
                         float *y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  y[i] = (float)(((hn[i] - h[i]) - ratio * (h[i] - hp[i])) * inv_s);
}

// guess: h_new = h + r (h - hp) + s o, corrections with |o| <= dead dropped (cells where
// the extrapolation is already right keep it exactly)
__global__ void k_apply_guess(int n, double *hn, const double *h, const double *hp, double ratio, double s,
                              const float *o, float dead) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float oi = o[i];
  hn[i] = h[i] + ratio * (h[i] - hp[i]) + ((fabsf(oi) > dead) ? s * (double)oi : 0.0);
}

__global__ void __launch_bounds__(256) k_sumsq_diff(int n, const double *a, const double *b, double *part) {
  __shared__ double sh[8];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = a[i] - b[i];
    s += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += sh[w];
    part[blockIdx.x] = t;
  }
}

// ---------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------
static int cnn_reserve(Net &n, int N) {
  if (n.cap >= N) return MSG_OK;
  for (int l = 0; l < kLayers; ++l) {
    if (n.a[l]) cudaFree(n.a[l]);
    if (n.z[l]) cudaFree(n.z[l]);
    MSG_CUDA(cudaMalloc(&n.a[l], (size_t)N * kC * 2));
    MSG_CUDA(cudaMalloc(&n.z[l], (size_t)N * kC * 4));
  }
  if (n.dz) cudaFree(n.dz);
  if (n.dz2) cudaFree(n.dz2);
  MSG_CUDA(cudaMalloc(&n.dz, (size_t)N * kC * 2));
  MSG_CUDA(cudaMalloc(&n.dz2, (size_t)N * kC * 2));
  int chunks = (N + kWgChunk - 1) / kWgChunk;
  if (n.part) cudaFree(n.part);
  n.part_cap = chunks;
  MSG_CUDA(cudaMalloc(&n.part, (size_t)chunks * kTaps * kC * kC * 4));
  n.cap = N;
  return MSG_OK;
}

static int cnn_forward(Net &n, const Grid3 &g, const __nv_bfloat16 *x) {
  cudaStream_t s = n.stream;
  int blocks = (g.N + 127) / 128;   // 8 warps x 16 cells
  const __nv_bfloat16 *in = x;
  for (int l = 0; l < kLayers - 1; ++l) {
    k_conv<0><<<blocks, 256, 0, s>>>(g, in, n.w16 + (size_t)l * kWl, n.w32 + (size_t)l * kPl + kWl, n.z[l],
                                     n.a[l + 1], nullptr, nullptr, nullptr);
    MSG_CHECK_LAUNCH();
    in = n.a[l + 1];
  }
  k_conv<1><<<blocks, 256, 0, s>>>(g, in, n.w16 + (size_t)3 * kWl, n.w32 + (size_t)3 * kPl + kWl, nullptr, nullptr,
                                   n.z[3], nullptr, nullptr);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

// backward from dz (channel 0 = dL/dout) at the output; grad filled
static int cnn_backward(Net &n, const Grid3 &g, const __nv_bfloat16 *x) {
  cudaStream_t s = n.stream;
  int blocks = (g.N + 127) / 128;
  int chunks = (g.N + kWgChunk - 1) / kWgChunk;
  __nv_bfloat16 *dz = n.dz, *dzn = n.dz2;
  for (int l = kLayers - 1; l >= 0; --l) {
    const __nv_bfloat16 *in = (l == 0) ? x : n.a[l];
    k_wgrad<<<dim3(chunks, kTaps), 128, 0, s>>>(g, dz, in, n.part);
    MSG_CHECK_LAUNCH();
    k_reduce_parts<<<(kWl + 255) / 256, 256, 0, s>>>(chunks, n.part, kWl, n.grad + (size_t)l * kPl);
    MSG_CHECK_LAUNCH();
    k_bgrad<<<chunks, 256, 0, s>>>(g, dz, n.part);
    MSG_CHECK_LAUNCH();
    k_reduce_parts<<<1, 32, 0, s>>>(chunks, n.part, kC, n.grad + (size_t)l * kPl + kWl);
    MSG_CHECK_LAUNCH();
    if (l > 0) {
      k_conv<2><<<blocks, 256, 0, s>>>(g, dz, n.wt16 + (size_t)l * kWl, nullptr, nullptr, nullptr, nullptr,
                                       n.z[l - 1], dzn);
      MSG_CHECK_LAUNCH();
      std::swap(dz, dzn);
    }
  }
  return MSG_OK;
}

static int cnn_loss(Net &n, const Grid3 &g, const float *y, double *loss) {
  double *part = nullptr;
  const int B = 296;
  MSG_CUDA(cudaMallocAsync(&part, B * 8, n.stream));
  k_loss<<<B, 256, 0, n.stream>>>(g.N, n.z[3], y, n.dz, part);
  MSG_CHECK_LAUNCH();
  std::vector<double> h(B);
  MSG_CUDA(cudaMemcpyAsync(h.data(), part, B * 8, cudaMemcpyDeviceToHost, n.stream));
  MSG_CUDA(cudaStreamSynchronize(n.stream));
  cudaFreeAsync(part, n.stream);
  double t = 0.0;
  for (double v : h) t += v;
  *loss = t / g.N;
  return MSG_OK;
}

static int cnn_pack(Net &n) {
  k_pack_weights<<<(kLayers * kWl + 255) / 256, 256, 0, n.stream>>>(n.w32, n.w16, n.wt16);
  MSG_CHECK_LAUNCH();
  return conv_pack_weights(n.w32, kPl, n.wtc, n.stream);
}

// Tensor-core forward pass from the plan's input buffer; *out = output channel (N floats).
static int cnn_forward_tc(Net &n, cudaStream_t s, const float **out, int withhold = -1) {
  const float *bias[kLayers];
  for (int l = 0; l < kLayers; ++l) bias[l] = n.w32 + (size_t)l * kPl + kWl;
  return conv_forward_tc(n.plan, n.wtc, bias, s, out, withhold);
}

static double host_sumsq_diff(msg_ctx *c, const double *a, const double *b, int *rc) {
  const int B = kRedBlocks;
  k_sumsq_diff<<<B, 256, 0, c->stream>>>(c->N, a, b, c->part);
  __atomic_fetch_add(&g_launches, 1LL, __ATOMIC_RELAXED);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("sumsq_diff launch: %s", cudaGetErrorString(e));
    *rc = MSG_ERR_CUDA;
    return 0.0;
  }
  double t = 0.0;
  *rc = finish(c, B, 1, &t);
  return t;
}

static FeatArgs feat_args(msg_ctx *c, double inv_s, double ratio) {
  FeatArgs f;
  f.g = Grid3{c->nx, c->ny, c->nz, c->nxy, c->N};
  f.h = c->head_old; f.hprev = c->head_old2; f.top = c->cell_top;
  f.ksz = c->ksz; f.reta = c->reta; f.retn = c->retn;
  f.calc_rech = c->calc_rech; f.rech_base = c->rech_base;
  f.len_scal = c->len_scal; f.inv_s = inv_s; f.ratio = ratio;
  return f;
}

bool learned_ready(msg_ctx *c) { return c->learned != nullptr; }

// Features of the current state and the tensor-core forward pass (no state change);
// *s_out / *ratio_out: the increment scale and the dt ratio the features were made with.
int learned_forward(msg_ctx *c, const float **out, double *s_out, double *ratio_out) {
  Net &n = reinterpret_cast<msg_cnn *>(c->learned)->net;
  std::lock_guard<std::recursive_mutex> lk(n.mu);
  int rc;
  double ss = host_sumsq_diff(c, c->head_old, c->head_old2, &rc);
  if (rc) return rc;
  double s = std::sqrt(ss / c->N) + 1e-30;
  double ratio = c->delt / c->delt_old1;
  if ((rc = conv_plan_get(&n.plan, c->nx, c->ny, c->nz))) return rc;
  k_features<true><<<(c->N + 255) / 256, 256, 0, c->stream>>>(feat_args(c, 1.0 / s, ratio), conv_plan_input(n.plan),
                                                               (long long)conv_plan_plane(n.plan));
  MSG_CHECK_LAUNCH();
  if ((rc = cnn_forward_tc(n, c->stream, out))) return rc;
  if (s_out) *s_out = s;
  if (ratio_out) *ratio_out = ratio;
  return MSG_OK;
}

int learned_convs(msg_ctx *c) {
  Net &n = reinterpret_cast<msg_cnn *>(c->learned)->net;
  std::lock_guard<std::recursive_mutex> lk(n.mu);
  const float *o = nullptr;
  return cnn_forward_tc(n, c->stream, &o);
}

int learned_check(msg_ctx *c) {
  Net &n = reinterpret_cast<msg_cnn *>(c->learned)->net;
  std::lock_guard<std::recursive_mutex> lk(n.mu);
  return conv_check(n.plan, c->stream);
}

// head_new <- h_old + r (h_old - h_old2) + s * CNN(features)
int learned_guess(msg_ctx *c) {
  Net &n = reinterpret_cast<msg_cnn *>(c->learned)->net;
  std::lock_guard<std::recursive_mutex> lk(n.mu);   // held until conv_check has synchronised
  const float *o = nullptr;
  double s = 0.0, ratio = 0.0;
  int rc = learned_forward(c, &o, &s, &ratio);
  if (rc) return rc;
  k_apply_guess<<<(c->N + 255) / 256, 256, 0, c->stream>>>(c->N, c->head_new, c->head_old, c->head_old2, ratio, s, o,
                                                          n.dead);
  MSG_CHECK_LAUNCH();
  return conv_check(n.plan, c->stream);
}

void learned_free(msg_ctx *c) { c->learned = nullptr; }   // the network is owned by its msg_cnn handle

}  // namespace msg

using namespace msg;

extern "C" {

MSG_API int msg_gpu_cnn_create(int32_t seed, msg_cnn_t **out) {
  if (!out) return MSG_ERR_ARG;
  msg_cnn *h = new msg_cnn();
  Net &n = h->net;
  MSG_CUDA(cudaStreamCreateWithFlags(&n.stream, cudaStreamNonBlocking));
  MSG_CUDA(cudaMalloc(&n.w32, kNParam * 4));
  MSG_CUDA(cudaMalloc(&n.m, kNParam * 4));
  MSG_CUDA(cudaMalloc(&n.v, kNParam * 4));
  MSG_CUDA(cudaMalloc(&n.grad, kNParam * 4));
  MSG_CUDA(cudaMalloc(&n.w16, kLayers * kWl * 2));
  MSG_CUDA(cudaMalloc(&n.wt16, kLayers * kWl * 2));
  MSG_CUDA(cudaMalloc(&n.wtc, conv_packed_elems() * 2));
  // every upload goes through the network's own (non-blocking) stream, so the kernels that
  // follow on that stream see it
  MSG_CUDA(cudaMemsetAsync(n.m, 0, kNParam * 4, n.stream));
  MSG_CUDA(cudaMemsetAsync(n.v, 0, kNParam * 4, n.stream));
  // He-style init on the real fan-in (27 x used input channels); last layer starts at zero
  std::vector<float> w(kNParam, 0.f);
  unsigned long long st = 0x9E3779B97F4A7C15ull ^ (unsigned long long)seed;
  auto rnd = [&]() {
    st ^= st << 13; st ^= st >> 7; st ^= st << 17;
    return (double)(st >> 11) * (1.0 / 9007199254740992.0);
  };
  const int cin[kLayers] = {7, 16, 16, 16}, cout[kLayers] = {16, 16, 16, 1};
  for (int l = 0; l < kLayers - 1; ++l) {
    double sd = std::sqrt(2.0 / (27.0 * cin[l]));
    for (int tap = 0; tap < kTaps; ++tap)
      for (int co = 0; co < cout[l]; ++co)
        for (int ci = 0; ci < cin[l]; ++ci) {
          double u1 = std::max(rnd(), 1e-12), u2 = rnd();
          w[(size_t)l * kPl + (size_t)tap * kC * kC + co * kC + ci] =
              (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
        }
  }
  MSG_CUDA(cudaMemcpyAsync(n.w32, w.data(), kNParam * 4, cudaMemcpyHostToDevice, n.stream));
  int rc = cnn_pack(n);
  if (rc) return rc;
  MSG_CUDA(cudaStreamSynchronize(n.stream));
  *out = h;
  return MSG_OK;
}

MSG_API void msg_gpu_cnn_destroy(msg_cnn_t *h) {
  if (!h) return;
  Net &n = h->net;
  cudaStreamSynchronize(n.stream);
  void *p[] = {n.w32, n.w16, n.wt16, n.wtc, n.m, n.v, n.grad, n.part, n.dz, n.dz2, n.loss_part};
  conv_plan_free(n.plan);
  for (void *q : p) if (q) cudaFree(q);
  for (int l = 0; l < kLayers; ++l) { if (n.a[l]) cudaFree(n.a[l]); if (n.z[l]) cudaFree(n.z[l]); }
  for (auto &smp : n.data) { cudaFree(smp.x); cudaFree(smp.y); }
  cudaStreamDestroy(n.stream);
  delete h;
}

MSG_API int msg_gpu_cnn_nparam(void) { return kNParam; }

MSG_API int msg_gpu_cnn_set_deadband(msg_cnn_t *h, float dead) {
  if (!h || !(dead >= 0.0f)) return MSG_ERR_ARG;
  h->net.dead = dead;
  return MSG_OK;
}

MSG_API int msg_gpu_cnn_get_weights(msg_cnn_t *h, float *w) {
  if (!h || !w) return MSG_ERR_ARG;
  MSG_CUDA(cudaStreamSynchronize(h->net.stream));
  MSG_CUDA(cudaMemcpy(w, h->net.w32, kNParam * 4, cudaMemcpyDeviceToHost));
  return MSG_OK;
}

MSG_API int msg_gpu_cnn_set_weights(msg_cnn_t *h, const float *w) {
  if (!h || !w) return MSG_ERR_ARG;
  MSG_CUDA(cudaMemcpyAsync(h->net.w32, w, kNParam * 4, cudaMemcpyHostToDevice, h->net.stream));
  int rc = cnn_pack(h->net);
  if (rc) return rc;
  MSG_CUDA(cudaStreamSynchronize(h->net.stream));
  return MSG_OK;
}

// Append one training sample from a context right after an accepted step:
// features from (head_old, head_old2, dt ratio), target from head_new.
MSG_API int msg_gpu_cnn_collect(msg_cnn_t *h, msg_ctx_t *c) {
  if (!h || !c) return MSG_ERR_ARG;
  if (c->timestep_num < 1) { set_error("cnn_collect: need two previous time levels"); return MSG_ERR_STATE; }
  int rc;
  double ss = host_sumsq_diff(c, c->head_old, c->head_old2, &rc);
  if (rc) return rc;
  double s = std::sqrt(ss / c->N);
  if (!(s > 0.0)) return MSG_OK;   // no motion: nothing to learn from this step
  double ratio = c->delt / c->delt_old1;
  Net &n = h->net;
  n.seen++;
  long long slot = -1;                       // -1: append
  if (n.store_cap > 0 && (long long)n.data.size() >= n.store_cap) {
    n.rs ^= n.rs << 13; n.rs ^= n.rs >> 7; n.rs ^= n.rs << 17;
    long long r = (long long)(n.rs % (unsigned long long)n.seen);
    if (r >= n.store_cap) return MSG_OK;     // not kept
    slot = r;
  }
  Sample smp;
  smp.g = Grid3{c->nx, c->ny, c->nz, c->nxy, c->N};
  if (slot >= 0 && n.data[slot].g.N == c->N) {
    smp.x = n.data[slot].x; smp.y = n.data[slot].y;       // same size: reuse the buffers
  } else {
    MSG_CUDA(cudaMalloc(&smp.x, (size_t)c->N * kC * 2));
    MSG_CUDA(cudaMalloc(&smp.y, (size_t)c->N * 4));
  }
  k_features<false><<<(c->N + 255) / 256, 256, 0, c->stream>>>(feat_args(c, 1.0 / s, ratio), smp.x, 0);
  MSG_CHECK_LAUNCH();
  k_target<<<(c->N + 255) / 256, 256, 0, c->stream>>>(c->N, c->head_new, c->head_old, c->head_old2, ratio, 1.0 / s,
                                                     smp.y);
  MSG_CHECK_LAUNCH();
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  if (slot < 0) {
    n.data.push_back(smp);
  } else {
    if (n.data[slot].x != smp.x) {
      MSG_CUDA(cudaStreamSynchronize(n.stream));        // training may still read the old one
      cudaFree(n.data[slot].x); cudaFree(n.data[slot].y);
    }
    n.data[slot] = smp;
  }
  return MSG_OK;
}

MSG_API int msg_gpu_cnn_nsamples(msg_cnn_t *h) { return h ? (int)h->net.data.size() : 0; }

// Bound the sample store to `cap` samples (0: unbounded) kept by reservoir sampling over the
// collected steps; `seed` seeds the replacement draws.  Existing samples are kept.
MSG_API int msg_gpu_cnn_set_capacity(msg_cnn_t *h, int32_t cap, int32_t seed) {
  if (!h || cap < 0) return MSG_ERR_ARG;
  h->net.store_cap = cap;
  h->net.seen = (long long)h->net.data.size();
  h->net.rs = 0x2545F4914F6CDD1Dull ^ ((unsigned long long)(seed + 1) * 0x9E3779B97F4A7C15ull);
  return MSG_OK;
}
// Steps offered to msg_gpu_cnn_collect since the capacity was set (kept or not).
MSG_API long long msg_gpu_cnn_seen(msg_cnn_t *h) { return h ? h->net.seen : 0; }

// Load a sample from host arrays (x: [N][16] float features, y: [N] target).
MSG_API int msg_gpu_cnn_add_sample(msg_cnn_t *h, int32_t nx, int32_t ny, int32_t nz, const float *x, const float *y) {
  if (!h || !x || !y || nx < 1 || ny < 1 || nz < 1) return MSG_ERR_ARG;
  Sample smp;
  smp.g = Grid3{nx, ny, nz, nx * ny, nx * ny * nz};
  size_t N = smp.g.N;
  std::vector<__nv_bfloat16> xb(N * kC);
  for (size_t k = 0; k < N * kC; ++k) xb[k] = __float2bfloat16(x[k]);
  MSG_CUDA(cudaMalloc(&smp.x, N * kC * 2));
  MSG_CUDA(cudaMalloc(&smp.y, N * 4));
  MSG_CUDA(cudaMemcpyAsync(smp.x, xb.data(), N * kC * 2, cudaMemcpyHostToDevice, h->net.stream));
  MSG_CUDA(cudaMemcpyAsync(smp.y, y, N * 4, cudaMemcpyHostToDevice, h->net.stream));
  MSG_CUDA(cudaStreamSynchronize(h->net.stream));
  h->net.data.push_back(smp);
  return MSG_OK;
}

// Loss (mean squared error) and optionally the gradient (host, kNParam floats) on one sample.
MSG_API int msg_gpu_cnn_loss_grad(msg_cnn_t *h, int32_t sample, double *loss, float *grad, float *out) {
  if (!h || sample < 0 || sample >= (int)h->net.data.size()) return MSG_ERR_ARG;
  Net &n = h->net;
  Sample &smp = n.data[sample];
  int rc;
  if ((rc = cnn_reserve(n, smp.g.N))) return rc;
  if ((rc = cnn_forward(n, smp.g, smp.x))) return rc;
  double L = 0.0;
  if ((rc = cnn_loss(n, smp.g, smp.y, &L))) return rc;
  if (loss) *loss = L;
  if (grad) {
    if ((rc = cnn_backward(n, smp.g, smp.x))) return rc;
    MSG_CUDA(cudaStreamSynchronize(n.stream));
    MSG_CUDA(cudaMemcpy(grad, n.grad, kNParam * 4, cudaMemcpyDeviceToHost));
  }
  if (out) {
    MSG_CUDA(cudaStreamSynchronize(n.stream));
    MSG_CUDA(cudaMemcpy(out, n.z[3], (size_t)smp.g.N * 4, cudaMemcpyDeviceToHost));
  }
  return MSG_OK;
}

// Inference pass of the tensor-core path on one stored sample: out = N floats.
static int cnn_infer(msg_cnn_t *h, int32_t sample, float *out, int withhold) {
  if (!h || !out || sample < 0 || sample >= (int)h->net.data.size()) return MSG_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(h->net.mu);
  Net &n = h->net;
  Sample &smp = n.data[sample];
  int rc;
  if ((rc = conv_plan_get(&n.plan, smp.g.nx, smp.g.ny, smp.g.nz))) return rc;
  if ((rc = conv_plan_load_compact(n.plan, smp.x, n.stream))) return rc;
  const float *o = nullptr;
  if ((rc = cnn_forward_tc(n, n.stream, &o, withhold))) return rc;
  if ((rc = conv_check(n.plan, n.stream))) return rc;
  MSG_CUDA(cudaMemcpy(out, o, (size_t)smp.g.N * 4, cudaMemcpyDeviceToHost));
  return MSG_OK;
}

MSG_API int msg_gpu_cnn_infer(msg_cnn_t *h, int32_t sample, float *out) { return cnn_infer(h, sample, out, -1); }

MSG_API int msg_gpu_cnn_infer_withhold(msg_cnn_t *h, int32_t sample, int32_t tile, float *out) {
  if (tile < 0) return MSG_ERR_ARG;
  return cnn_infer(h, sample, out, tile);
}

// `iters` AdamW steps over the stored samples (sample order from `seed`); returns the
// mean loss of the last epoch-sized window.
MSG_API int msg_gpu_cnn_train(msg_cnn_t *h, int32_t iters, float lr, float weight_decay, int32_t seed,
                              double *mean_loss) {
  if (!h || iters < 0) return MSG_ERR_ARG;
  Net &n = h->net;
  int ns = (int)n.data.size();
  if (ns == 0) { set_error("cnn_train: no samples"); return MSG_ERR_STATE; }
  int maxN = 0;
  for (auto &smp : n.data) maxN = std::max(maxN, smp.g.N);
  int rc;
  if ((rc = cnn_reserve(n, maxN))) return rc;
  unsigned long long st = 88172645463325252ull ^ (unsigned long long)(seed + 1);
  double acc = 0.0;
  int cnt = 0;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int it = 0; it < iters; ++it) {
    st ^= st << 13; st ^= st >> 7; st ^= st << 17;
    Sample &smp = n.data[st % ns];
    if ((rc = cnn_forward(n, smp.g, smp.x))) return rc;
    double L = 0.0;
    if ((rc = cnn_loss(n, smp.g, smp.y, &L))) return rc;
    if ((rc = cnn_backward(n, smp.g, smp.x))) return rc;
    n.step++;
    float c1 = 1.f - std::pow(b1, (float)n.step), c2 = 1.f - std::pow(b2, (float)n.step);
    k_adamw<<<(kNParam + 255) / 256, 256, 0, n.stream>>>(kNParam, n.w32, n.grad, n.m, n.v, lr, b1, b2, eps,
                                                         weight_decay, c1, c2);
    MSG_CHECK_LAUNCH();
    if ((rc = cnn_pack(n))) return rc;
    if (it >= iters - std::max(1, std::min(iters, ns))) { acc += L; cnt++; }
  }
  MSG_CUDA(cudaStreamSynchronize(n.stream));
  if (mean_loss) *mean_loss = cnt ? acc / cnt : 0.0;
  return MSG_OK;
}

// Use this network for guess_mode = 2 in the context (NULL detaches).
MSG_API int msg_gpu_cnn_attach(msg_ctx_t *c, msg_cnn_t *h) {
  if (!c) return MSG_ERR_ARG;
  c->learned = h;
  return MSG_OK;
}

MSG_API int msg_gpu_guess_fallbacks(msg_ctx_t *c) { return c ? c->guess_fallbacks : 0; }
MSG_API int msg_gpu_guess_rejected(msg_ctx_t *c) { return c ? c->guess_rejected : 0; }

}  // extern "C"
