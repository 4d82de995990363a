// msg_conv_tc.cu -- implicit-GEMM 3x3x3 convolution of the learned-guess CNN on the
// 5th-generation tensor cores (tcgen05.mma, accumulators in tensor memory, TMA staging).
//
// One tile = 8 (x) x 16 (y) cells of one z plane (the GEMM M = 128, row m = 8 y + x).
// The activations are kept halo-padded and chunk-planar (msg_conv_tc.cuh), and the TMA
// map flattens (x, channel) of a chunk plane into its innermost dimension, so the halo
// block of a tile -- 10 cells x 18 rows x 3 planes x 2 chunks -- arrives as ONE 4-D box of
// 17,280 B made of 160-B rows.  In shared memory the box is exactly the K-major
// no-swizzle operand layout: a core matrix is the 8 x cells of one row (16 B each), the
// 8-row groups (y) are 160 B apart, the two channel chunks 8,640 B apart.  The A operand
// of each of the 27 taps is therefore a shifted view of the box -- only the start address
// of the matrix descriptor moves (16 B per x step, 160 B per y step, 2,880 B per z step).
// Nothing is re-staged per tap and no boundary test is made: the zero halo is the
// convolution's zero padding, and the TMA zero-fills past the grid.
// B = the tap's 16 x 16 weights; D (128 x 16 FP32) accumulates in TMEM over the 27 taps
// (27 x tcgen05.mma M128 N16 K16, BF16 inputs), alternating between kChains accumulators
// (summed in the epilogue) so that successive MMAs do not wait on one accumulator.
//
// Warp roles (192 threads, three persistent CTAs per SM, 67 KB of shared memory each):
//   warp 0      TMA producer over a 3-stage ring; allocates and frees the TMEM columns
//   warp 1      MMA issuer (one thread); commits each tile to the stage's "empty" barrier
//               and to the accumulator's "full" barrier
//   warps 2-5   epilogue: tcgen05.ld of the accumulators (double-buffered), bias, GELU,
//               BF16, stores into the next layer's padded buffer
// Every mbarrier wait is bounded (one second on %globaltimer).  On expiry the CTA records an
// error code, stops issuing, waits (bounded) for the copies and MMAs it issued, frees TMEM
// and returns; the host reads the code after the pass.
#include "msg_conv_tc.cuh"
#include <cuda.h>
#include <cudaTypedefs.h>
#include <mutex>

namespace msg {

namespace {
constexpr int kCh = 16, kNTaps = 27, kNLayers = 4;
constexpr int kTX = 8, kTY = 16, kTM = kTX * kTY;       // tile: 8 x 16 cells (GEMM M = 128)
constexpr int kBX = kTX + 2, kBY = kTY + 2;              // halo block: 10 cells x 18 rows x 3 planes
constexpr int kRowBytes = kBX * 16;                      // one chunk of one halo row: 160 B
constexpr int kPlaneBytes = kBY * kRowBytes;             // one chunk of one plane: 2880 B
constexpr int kChunkBytes = 3 * kPlaneBytes;             // one chunk of the block: 8640 B
constexpr int kBoxBytes = 2 * kChunkBytes;               // bytes one TMA box delivers: 17280
constexpr int kStageBytes = 17408;                       // stage pitch, a multiple of 128 B
constexpr int kStages = 3;
constexpr int kTapBytes = 512;                           // 16 co x 16 ci, BF16
constexpr int kWBytes = kNTaps * kTapBytes;              // 13824 B
constexpr int kCtl = kStages * kStageBytes + kWBytes;    // control block offset (66048)
constexpr int kSmemTC = kCtl + 256 + 1024;               // + barriers + alignment slack
constexpr int kThreadsTC = 192;
constexpr int kCtaPerSm = 3;
constexpr int kChains = 2;                               // independent accumulators per tile (taps mod 2)
constexpr int kAccCols = kChains * 16;                   // TMEM columns of one accumulator set
constexpr int kTmemCols = 2 * kAccCols;                  // double-buffered: 64 columns
constexpr unsigned long long kWaitNs = 1000000000ull;    // bound on every wait
static_assert(kStageBytes >= kBoxBytes && kStageBytes % 128 == 0, "stage pitch");
static_assert(kCtl % 128 == 0, "control block alignment");
static_assert(kTmemCols >= 32 && (kTmemCols & (kTmemCols - 1)) == 0, "TMEM allocation is a power of 2 >= 32");
}  // namespace

struct ConvPlan {
  CUtensorMap map[3];                 // TMA maps of buf[0..2]
  int nx = 0, ny = 0, nz = 0, px = 0, py = 0, pz = 0, device = -1, nsm = 148;
  long long plane = 0;                // padded cells per chunk plane
  __nv_bfloat16 *buf[3] = {nullptr, nullptr, nullptr};   // input features, two hidden ping-pong buffers
  float *out = nullptr;               // output channel, interior order
  int *err = nullptr;
  int *err_host = nullptr;
};

struct TcArgs {
  int nx, ny, px, py, ntx, nty, ntiles;
  long long plane;
  const __nv_bfloat16 *w;    // packed weights of this layer (27 x 512 B)
  const float *bias;         // 16 floats
  __nv_bfloat16 *act_out;    // hidden layer output (padded, chunk-planar)
  float *out;                // output layer: channel 0, interior order
  int *err;
  int withhold;              // test hook: the box of this tile is never loaded (-1: none)
};

// ---------------------------------------------------------------------------------
// PTX wrappers
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// One try_wait with a suspend-time hint: the thread sleeps in hardware until the phase
// completes or about `hint_ns` have passed (no busy spinning).
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0u;
}

// Wait for the phase of parity `parity`; false after kWaitNs or when *abort_flag is set.
// The timer is read once per 64 sleeps of at most 1 ms each.
__device__ __noinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag) {
  if (mbar_test(bar, parity, 1000000u)) return true;
  const unsigned long long t0 = gtime();
  for (unsigned k = 1;; ++k) {
    if (mbar_test(bar, parity, 1000000u)) return true;
    if (abort_flag && *abort_flag) return false;
    if ((k & 63u) == 0u && gtime() - t0 > kWaitNs) return false;
  }
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
      "[%2];" ::"r"(dst),
      "l"((unsigned long long)map), "r"(bar), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}

// Shared-memory matrix descriptor, no swizzle, K-major: 8-row x 16-B core matrices,
// `lbo` bytes between the two K halves, `sbo` bytes between 8-row groups.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 TMEM lanes (this warp's sub-partition) x 16 FP32 columns -> 16 values per thread.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  // the registers are defined only after the wait: thread them through it
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu_tc(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

// ---------------------------------------------------------------------------------
// the convolution kernel
// MODE 0: hidden layer -> bias + GELU -> BF16 into the padded output buffer
// MODE 1: output layer -> channel 0 + bias into out[] (interior order)
// ---------------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(kThreadsTC, kCtaPerSm) k_conv_tc(const __grid_constant__ CUtensorMap in_map, TcArgs a) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = su32(sm);
  const uint32_t wsm = sbase + kStages * kStageBytes;
  unsigned char *ctl = sm + kCtl;
  const uint32_t cb = su32(ctl);
  // barriers: full[4] @0, empty[4] @32, acc_full[2] @64, acc_empty[2] @80, drain @96
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(ctl + 112);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(ctl + 120);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // weights -> shared memory (generic proxy), then made visible to the async proxy
  for (int k = threadIdx.x; k < kWBytes / 16; k += blockDim.x)
    reinterpret_cast<uint4 *>(sm + kStages * kStageBytes)[k] = reinterpret_cast<const uint4 *>(a.w)[k];
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(cb + 8 * s, 1);
      mbar_init(cb + 32 + 8 * s, 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(cb + 64 + 8 * b, 1);
      mbar_init(cb + 80 + 8 * b, 4);
    }
    mbar_init(cb + 96, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                 "n"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer ----
      int j = 0, withheld = -1;
      for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++j) {
        const int s = j % kStages;
        if (!mbar_wait(cb + 32 + 8 * s, ((j / kStages) & 1) ^ 1, abort_flag)) {
          atomicCAS(a.err, 0, 1);
          *abort_flag = 1;
          break;
        }
        if (t == a.withhold) {   // the consumer's bounded wait on this stage runs out
          withheld = j;
          continue;
        }
        const int tx = t % a.ntx, r = t / a.ntx, ty = r % a.nty, z = r / a.nty;
        mbar_expect_tx(cb + 8 * s, kBoxBytes);
        // box origin in padded coordinates = interior (x0 - 1, y0 - 1, z - 1); the innermost
        // coordinate counts BF16 elements of the flattened (x, channel) row: 8 per cell
        tma_load_4d(sbase + s * kStageBytes, &in_map, cb + 8 * s, 8 * kTX * tx, kTY * ty, z, 0);
      }
      // every issued box must have landed before the CTA may exit
      for (int q = (j > kStages ? j - kStages : 0); q < j; ++q)
        if (q != withheld && !mbar_wait(cb + 8 * (q % kStages), (q / kStages) & 1, nullptr)) atomicCAS(a.err, 0, 5);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer (one thread) ----
      // kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major, N = 16, M = 128
      constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kCh >> 3) << 17) |
                                 ((uint32_t)(kTM >> 4) << 24);
      const uint64_t bdesc0 = sdesc(wsm, 256, 128);
      int j = 0;
      for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++j) {
        const int s = j % kStages, b = j & 1;
        if (!mbar_wait(cb + 8 * s, (j / kStages) & 1, abort_flag) ||
            !mbar_wait(cb + 80 + 8 * b, ((j >> 1) & 1) ^ 1, abort_flag)) {
          atomicCAS(a.err, 0, 2);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint64_t adesc0 = sdesc(sbase + s * kStageBytes, kChunkBytes, kRowBytes);
        const uint32_t d0 = tmem + b * kAccCols;
        // fully unrolled: tap (dx, dy, dz) = (tap % 3, tap / 3 % 3, tap / 9) is a compile-time
        // shift of the A start address (descriptor field in 16-B units); B = the tap's
        // 512-B weight block.  The issue loop is then descriptor adds and MMAs only.
#pragma unroll
        for (int tap = 0; tap < kNTaps; ++tap) {
          const uint64_t ad = adesc0 + (uint64_t)(((tap % 3) * 16 + ((tap / 3) % 3) * kRowBytes + (tap / 9) * kPlaneBytes) >> 4);
          const uint64_t bd = bdesc0 + (uint64_t)((tap * kTapBytes) >> 4);
          umma_bf16(d0 + (tap % kChains) * kCh, ad, bd, idesc, tap >= kChains ? 1u : 0u);
        }
        umma_commit(cb + 32 + 8 * s);   // stage s free once these MMAs have read it
        umma_commit(cb + 64 + 8 * b);   // accumulator b ready
      }
      umma_commit(cb + 96);             // all MMAs of this CTA done
      if (!mbar_wait(cb + 96, 0, nullptr)) atomicCAS(a.err, 0, 6);
    }
  } else {
    // ---- epilogue: warps 2..5 own TMEM sub-partitions 2, 3, 0, 1 ----
    const int sub = warp & 3;
    const int row = sub * 32 + lane;
    const int xx = row % kTX, yy = row / kTX;
    float bias[kCh];
#pragma unroll
    for (int c = 0; c < kCh; ++c) bias[c] = a.bias[c];
    int j = 0;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++j) {
      const int b = j & 1;
      // one lane per warp waits; the others join it at the vote
      bool ok = true;
      if (lane == 0) ok = mbar_wait(cb + 64 + 8 * b, (j >> 1) & 1, abort_flag);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) {
          atomicCAS(a.err, 0, 3);
          *abort_flag = 1;
        }
        break;
      }
      tc_fence_after();
      float v[kCh];
      const uint32_t tb = tmem + ((uint32_t)(sub * 32) << 16) + (uint32_t)(b * kAccCols);
      tmem_ld16(tb, v);
#pragma unroll
      for (int c = 1; c < kChains; ++c) {
        float w[kCh];
        tmem_ld16(tb + c * kCh, w);
#pragma unroll
        for (int q = 0; q < kCh; ++q) v[q] += w[q];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(cb + 80 + 8 * b);
      const int tx = t % a.ntx, r = t / a.ntx, ty = r % a.nty, z = r / a.nty;
      const int x = tx * kTX + xx, y = ty * kTY + yy;
      if (x < a.nx && y < a.ny) {
        if (MODE == 0) {
          __align__(16) __nv_bfloat16 o[kCh];
#pragma unroll
          for (int c = 0; c < kCh; ++c) o[c] = __float2bfloat16(gelu_tc(v[c] + bias[c]));
          const long long p = ((long long)(z + 1) * a.py + (y + 1)) * a.px + (x + 1);
          uint4 *dst = reinterpret_cast<uint4 *>(a.act_out);
          dst[p] = reinterpret_cast<const uint4 *>(o)[0];
          dst[a.plane + p] = reinterpret_cast<const uint4 *>(o)[1];
        } else {
          a.out[((long long)z * a.ny + y) * a.nx + x] = v[0] + bias[0];
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(kTmemCols) : "memory");
  }
}

// ---------------------------------------------------------------------------------
// layout helpers
// ---------------------------------------------------------------------------------
__global__ void k_pack_tc(const float *w32, int lstride, __nv_bfloat16 *wpk) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;   // [layer][tap][k chunk][co][8 ci]
  if (e >= kNLayers * kNTaps * 256) return;
  int l = e / (kNTaps * 256), r = e - l * (kNTaps * 256);
  int tap = r / 256, q = r % 256;
  int kc = q / 128, co = (q / 8) % 16, ci = kc * 8 + q % 8;
  wpk[e] = __float2bfloat16(w32[(size_t)l * lstride + (size_t)(tap * kCh + co) * kCh + ci]);
}

__global__ void k_compact_to_pad(int nx, int ny, int nz, int px, int py, long long plane, const uint4 *x, uint4 *buf) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long N = (long long)nx * ny * nz;
  if (i >= N) return;
  int iz = (int)(i / ((long long)nx * ny)), rem = (int)(i - (long long)iz * nx * ny), iy = rem / nx, ix = rem - iy * nx;
  long long p = ((long long)(iz + 1) * py + (iy + 1)) * px + (ix + 1);
  buf[p] = x[2 * i];
  buf[plane + p] = x[2 * i + 1];
}

// ---------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

void conv_plan_free(ConvPlan *p) {
  if (!p) return;
  for (auto *b : p->buf) if (b) cudaFree(b);
  if (p->out) cudaFree(p->out);
  if (p->err) cudaFree(p->err);
  if (p->err_host) cudaFreeHost(p->err_host);
  delete p;
}

int conv_plan_get(ConvPlan **plan, int nx, int ny, int nz) {
  int dev = 0;
  MSG_CUDA(cudaGetDevice(&dev));
  ConvPlan *p = *plan;
  if (p && p->nx == nx && p->ny == ny && p->nz == nz && p->device == dev) return MSG_OK;
  conv_plan_free(p);
  *plan = nullptr;
  auto fn = encode_fn();
  if (!fn) {
    set_error("conv_plan: cuTensorMapEncodeTiled is not available from the driver");
    return MSG_ERR_CUDA;
  }
  p = new ConvPlan();
  p->nx = nx; p->ny = ny; p->nz = nz; p->device = dev;
  p->px = nx + 2; p->py = ny + 2; p->pz = nz + 2;
  p->plane = (long long)p->px * p->py * p->pz;
  MSG_CUDA(cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, dev));
  const size_t bytes = (size_t)p->plane * 2 * 16;
  for (int k = 0; k < 3; ++k) {
    MSG_CUDA(cudaMalloc(&p->buf[k], bytes));
    MSG_CUDA(cudaMemset(p->buf[k], 0, bytes));   // the halo stays zero from here on
    // dims: (x, channel) flattened, y, z, chunk
    cuuint64_t dims[4] = {8ull * p->px, (cuuint64_t)p->py, (cuuint64_t)p->pz, 2};
    cuuint64_t strides[3] = {16ull * p->px, 16ull * p->px * p->py, 16ull * (cuuint64_t)p->plane};
    cuuint32_t box[4] = {8u * kBX, (cuuint32_t)kBY, 3, 2};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = fn(&p->map[k], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, p->buf[k], dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      set_error("conv_plan: cuTensorMapEncodeTiled failed (%d) for %dx%dx%d", (int)r, nx, ny, nz);
      conv_plan_free(p);
      return MSG_ERR_CUDA;
    }
  }
  MSG_CUDA(cudaMalloc(&p->out, (size_t)nx * ny * nz * 4));
  MSG_CUDA(cudaMalloc(&p->err, 4));
  MSG_CUDA(cudaMallocHost(&p->err_host, 4));
  *plan = p;
  return MSG_OK;
}

__nv_bfloat16 *conv_plan_input(ConvPlan *p) { return p->buf[0]; }
size_t conv_plan_plane(ConvPlan *p) { return (size_t)p->plane; }

int conv_plan_load_compact(ConvPlan *p, const __nv_bfloat16 *x, cudaStream_t s) {
  long long N = (long long)p->nx * p->ny * p->nz;
  k_compact_to_pad<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(p->nx, p->ny, p->nz, p->px, p->py, p->plane,
                                                              reinterpret_cast<const uint4 *>(x),
                                                              reinterpret_cast<uint4 *>(p->buf[0]));
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int conv_pack_weights(const float *w32, int layer_stride, __nv_bfloat16 *wpk, cudaStream_t s) {
  k_pack_tc<<<(kNLayers * kNTaps * 256 + 255) / 256, 256, 0, s>>>(w32, layer_stride, wpk);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int conv_forward_tc(ConvPlan *p, const __nv_bfloat16 *wpk, const float *const bias[4], cudaStream_t s,
                    const float **out, int withhold) {
  TcArgs a;
  a.withhold = withhold;
  a.nx = p->nx; a.ny = p->ny; a.px = p->px; a.py = p->py;
  a.ntx = (p->nx + kTX - 1) / kTX;
  a.nty = (p->ny + kTY - 1) / kTY;
  a.ntiles = a.ntx * a.nty * p->nz;
  a.plane = p->plane;
  a.out = p->out;
  a.err = p->err;
  const int grid = a.ntiles < kCtaPerSm * p->nsm ? a.ntiles : kCtaPerSm * p->nsm;
  MSG_CUDA(cudaFuncSetAttribute(k_conv_tc<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTC));
  MSG_CUDA(cudaFuncSetAttribute(k_conv_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTC));
  MSG_CUDA(cudaMemsetAsync(p->err, 0, 4, s));
  int in = 0, nxt = 1;
  for (int l = 0; l < kNLayers; ++l) {
    a.w = wpk + (size_t)l * kNTaps * 256;
    a.bias = bias[l];
    if (l < kNLayers - 1) {
      a.act_out = p->buf[nxt];
      k_conv_tc<0><<<grid, kThreadsTC, kSmemTC, s>>>(p->map[in], a);
      MSG_CHECK_LAUNCH();
      a.withhold = -1;
      in = nxt;
      nxt = (nxt == 1) ? 2 : 1;
    } else {
      a.act_out = nullptr;
      k_conv_tc<1><<<grid, kThreadsTC, kSmemTC, s>>>(p->map[in], a);
      MSG_CHECK_LAUNCH();
    }
  }
  MSG_CUDA(cudaMemcpyAsync(p->err_host, p->err, 4, cudaMemcpyDeviceToHost, s));
  *out = p->out;
  return MSG_OK;
}

// Status of the last forward pass (synchronises the stream).
int conv_check(ConvPlan *p, cudaStream_t s) {
  MSG_CUDA(cudaStreamSynchronize(s));
  if (*p->err_host) {
    set_error("tensor-core convolution: a bounded wait ran out (code %d: 1 producer, 2 MMA issuer, 3 epilogue, "
              "5 copy drain, 6 MMA drain)", *p->err_host);
    return MSG_ERR_CUDA;
  }
  return MSG_OK;
}

}  // namespace msg
