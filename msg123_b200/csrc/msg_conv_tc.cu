// msg_conv_tc.cu -- implicit-GEMM 3x3x3 convolution of the learned-guess CNN on the
// 5th-generation tensor cores (tcgen05.mma, accumulators in tensor memory, TMA staging).
//
// The GEMM's M = 128 rows are the cells of an 8 (x) x 16 (y) tile of one plane (row
// m = 8 y + x).  A CTA walks such a tile down z, one input plane at a time, over a segment
// of up to 32 output planes.  The activations are kept halo-padded and chunk-planar
// (msg_conv_tc.cuh), and the TMA map flattens (x, channel) of a chunk plane into its
// innermost dimension, so the input plane's halo block -- 10 cells x 18 rows x 2 channel
// chunks -- arrives as ONE 4-D box of 5,760 B made of 160-B rows.  In shared memory the box
// is exactly the K-major no-swizzle operand layout: a core matrix is the 8 x cells of one
// row (16 B each), 8-row groups (y) 160 B apart, the two chunks 2,880 B apart.  The A
// operand of each of the 9 in-plane taps (dx, dy) is a shifted view of the box -- only the
// start address of the matrix descriptor moves (16 B per x step, 160 B per y step).  The
// zero halo is the convolution's zero padding, and the TMA zero-fills past the grid.
//
// An input plane p feeds the output planes p+1, p and p-1 (taps dz = -1, 0, +1), so each
// in-plane tap is ONE tcgen05.mma M128 N48 K16 whose B holds the tap's 16 x 16 weights for
// all three (48 columns) and whose D is three 16-column accumulator slots in TMEM, output
// plane u (counted from the segment's start) in slot u mod 3.  The slots' roles rotate
// with the plane, so B is packed in three column rotations.  Once plane p's 9 MMAs are
// done, output plane p-1 has all 27 taps: the epilogue reads its slot, clears it for the
// plane it will hold next, and frees it.  Per plane: 9 MMAs and a 5.8-KB box (a tile-per-
// plane form needs 27 MMAs of N = 16 and a 17-KB three-plane box).
//
// Warp roles (192 threads, three persistent CTAs per SM, 71 KB of shared memory each):
//   warp 0      TMA producer over a 5-stage ring; allocates and frees the TMEM columns
//   warp 1      MMA issuer (one thread); commits each plane to the stage's "empty" barrier
//               and the completed output's slot to its "full" barrier
//   warps 2-5   epilogue: tcgen05.ld of the completed slot, clear, bias, GELU, BF16, stores
//               into the next layer's padded buffer
// A CTA runs two segments at once (two sets of three slots) and alternates their planes,
// so that one segment's MMAs proceed while the epilogue drains the other's.
// Every mbarrier wait is bounded (one second on %globaltimer).  On expiry the CTA records an
// error code, stops issuing, waits (bounded) for the copies and MMAs it issued, frees TMEM
// and returns; the host reads the code after the pass.
#include "msg_conv_tc.cuh"
#include <cuda.h>
#include <cudaTypedefs.h>
#include <mutex>

namespace msg {

namespace {
constexpr int kCh = 16, kNLayers = 4;
constexpr int kTX = 8, kTY = 16, kTM = kTX * kTY;       // tile: 8 x 16 cells (GEMM M = 128)
constexpr int kBX = kTX + 2, kBY = kTY + 2;              // halo block: 10 cells x 18 rows
constexpr int kRowBytes = kBX * 16;                      // one chunk of one halo row: 160 B
constexpr int kPlaneBytes = kBY * kRowBytes;             // one chunk of one plane: 2880 B
constexpr int kThreadsTC = 192;
constexpr int kCtaPerSm = 4;
constexpr unsigned long long kWaitNs = 1000000000ull;    // bound on every wait
constexpr int kZS = 32;                                  // output planes per segment of a column
constexpr int kBoxZ = 2 * kPlaneBytes;                   // one plane, two channel chunks: 5760 B
// Two input stages per CTA and four CTAs per SM (80 registers, 54 KB of shared memory and
// 128 TMEM columns each: the SM's 512 columns exactly) took the four layers at 25.2M cells
// from 3.98 ms (five stages, three CTAs per SM) to 3.27 ms; three stages at three CTAs gave
// 3.46 ms.  The results are the same bits.
constexpr int kStagesZ = 2;
constexpr int kStageZ = 5760;                            // a multiple of 128 B
constexpr int kNZ = 3 * kCh;                             // N = 48: three output planes of 16 channels
constexpr int kTapZ = 2 * kNZ * 16;                      // 48 co x 16 ci, BF16: 1536 B
constexpr int kWZ = 3 * 9 * kTapZ;                       // three rotations x 9 in-plane taps: 41472 B
constexpr int kCtlZ = kStagesZ * kStageZ + kWZ;          // 52992
constexpr int kSmemZ = kCtlZ + 256 + 1024;
constexpr int kTmemZ = 128;                              // two streams x 64 columns (48 used)
static_assert(kStageZ >= kBoxZ && kStageZ % 128 == 0 && kCtlZ % 128 == 0, "z-march layout");
static_assert(kCtaPerSm * (kSmemZ + 1024) <= 228 * 1024, "four CTAs per SM");
}  // namespace

struct ConvPlan {
  CUtensorMap map1[3];                // TMA maps of buf[0..2], one-plane boxes
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
// 32 TMEM lanes x 16 FP32 columns <- zero (clears an accumulator slot after it is read).
__device__ __forceinline__ void tmem_zero16(uint32_t taddr) {
  const uint32_t z = 0u;
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
      "%1};" ::"r"(taddr), "r"(z)
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// Work items of the z-march kernel.  A segment is one 8 x 16 column of the grid over kZS
// output planes [z0, z1); its items are the input planes z0-1 .. z1 (q = 0 .. L+1, the
// planes outside the grid being the buffer's zero halo).  A CTA takes segments
// blockIdx.x, +gridDim.x, ...; the even ones form stream 0, the odd ones stream 1, and the
// two streams' items alternate (while both have items), so that one stream's MMAs run while
// the epilogue drains the other's accumulators.  Producer, MMA issuer and epilogue walk the
// same sequence.
struct ZmIter {
  int nseg, nzs, nz, gstride;
  int seg[2], q[2], L[2];     // current segment (or -1), its item, its length
  int turn;
  __device__ void init(int first, int stride, int nseg_, int nzs_, int nz_) {
    nseg = nseg_; nzs = nzs_; nz = nz_; gstride = stride;
    for (int g = 0; g < 2; ++g) {
      const int sg = first + g * stride;
      seg[g] = sg < nseg ? sg : -1;
      q[g] = 0;
      L[g] = seg[g] >= 0 ? len(seg[g]) : 0;
    }
    turn = 0;
  }
  __device__ int len(int sg) const {
    const int z0 = (sg % nzs) * kZS;
    return min(kZS, nz - z0);
  }
  // next item: stream g, segment, q; false when both streams are done
  __device__ bool next(int &g, int &sg, int &qq, int &LL) {
    for (int k = 0; k < 2; ++k) {
      const int c = turn ^ k;
      if (seg[c] >= 0) {
        g = c; sg = seg[c]; qq = q[c]; LL = L[c];
        if (++q[c] > L[c] + 1) {   // segment done: the stream's next one
          const int nx = seg[c] + 2 * gstride;
          seg[c] = nx < nseg ? nx : -1;
          q[c] = 0;
          L[c] = seg[c] >= 0 ? len(seg[c]) : 0;
        }
        turn = c ^ 1;
        return true;
      }
    }
    return false;
  }
};

// The convolution marching down z.  For input plane p (q = p - z0 + 1 within its
// segment) every in-plane tap (dx, dy) is ONE tcgen05.mma with N = 48: A is the shifted
// view of the plane's halo box, B holds the tap's weights for the three output planes the
// plane feeds (p+1, p, p-1 through the taps dz = -1, 0, +1), and D is the stream's three
// accumulator slots of 16 columns, output plane u (= z - z0 + 1) in slot u mod 3.  The
// slots' roles rotate with q, so B comes in three column rotations (r = q mod 3).  After
// input q, output u = q - 1 has all its contributions: the epilogue reads it, clears its
// slot (it becomes output u + 3, started by input q + 2) and frees it.  Outputs u = -1, 0,
// L+1, L+2 of a segment (planes outside it) are computed and dropped.  Per plane: 9 MMAs
// and one 5.8-KB box instead of 27 MMAs and a 17-KB box.
template <int MODE>
__global__ void __launch_bounds__(kThreadsTC, kCtaPerSm) k_conv_zm(const __grid_constant__ CUtensorMap in_map, TcArgs a,
                                                                 int nseg, int nzs, int nz) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = su32(sm);
  const uint32_t wsm = sbase + kStagesZ * kStageZ;
  unsigned char *ctl = sm + kCtlZ;
  const uint32_t cb = su32(ctl);
  // barriers: full[5] @0, empty[5] @40, ofull[2][3] @80, oempty[2][3] @128, drain @176
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(ctl + 184);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(ctl + 188);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t FULL = cb, EMPTY = cb + 40, OFULL = cb + 80, OEMPTY = cb + 128, DRAIN = cb + 176;

  for (int k = threadIdx.x; k < kWZ / 16; k += blockDim.x)
    reinterpret_cast<uint4 *>(sm + kStagesZ * kStageZ)[k] = reinterpret_cast<const uint4 *>(a.w)[k];
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagesZ; ++s) {
      mbar_init(FULL + 8 * s, 1);
      mbar_init(EMPTY + 8 * s, 1);
    }
    for (int k = 0; k < 6; ++k) {
      mbar_init(OFULL + 8 * k, 1);
      mbar_init(OEMPTY + 8 * k, 4);
    }
    mbar_init(DRAIN, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tmem_slot)),
                 "n"(kTmemZ)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer: one single-plane box per item ----
      ZmIter it;
      it.init(blockIdx.x, gridDim.x, nseg, nzs, nz);
      int j = 0, withheld = -1, g, sg, q, L;
      while (it.next(g, sg, q, L)) {
        const int s = j % kStagesZ;
        if (!mbar_wait(EMPTY + 8 * s, ((j / kStagesZ) & 1) ^ 1, abort_flag)) {
          atomicCAS(a.err, 0, 1);
          *abort_flag = 1;
          break;
        }
        if (sg == a.withhold && q == 0 && withheld < 0) {   // the MMA issuer's bounded wait runs out
          withheld = j;
          ++j;
          continue;
        }
        const int col = sg / nzs, z0 = (sg % nzs) * kZS;
        const int tx = col % a.ntx, ty = col / a.ntx;
        mbar_expect_tx(FULL + 8 * s, kBoxZ);
        // padded plane index of input plane p = z0 - 1 + q is p + 1 = z0 + q
        tma_load_4d(sbase + s * kStageZ, &in_map, FULL + 8 * s, 8 * kTX * tx, kTY * ty, z0 + q, 0);
        ++j;
      }
      for (int k = (j > kStagesZ ? j - kStagesZ : 0); k < j; ++k)
        if (k != withheld && !mbar_wait(FULL + 8 * (k % kStagesZ), (k / kStagesZ) & 1, nullptr)) atomicCAS(a.err, 0, 5);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer ----
      // kind::f16: D FP32, A and B BF16, K-major, N = 48, M = 128
      constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kNZ >> 3) << 17) |
                                 ((uint32_t)(kTM >> 4) << 24);
      int nuse[2][3] = {{0, 0, 0}, {0, 0, 0}};
      ZmIter it;
      it.init(blockIdx.x, gridDim.x, nseg, nzs, nz);
      int j = 0, g, sg, q, L;
      bool bad = false;
      while (it.next(g, sg, q, L)) {
        const int s = j % kStagesZ;
        if (!mbar_wait(FULL + 8 * s, (j / kStagesZ) & 1, abort_flag)) { bad = true; break; }
        // slots this input starts: all three at q = 0, else the one of output q + 1
        for (int k = 0; k < 3; ++k) {
          const int sl = (q + 1 + 3 - k) % 3;   // k = 0: output q + 1; k = 1, 2: outputs q, q - 1
          if (k > 0 && q > 0) break;
          if (nuse[g][sl] > 0 && !mbar_wait(OEMPTY + 8 * (3 * g + sl), (nuse[g][sl] - 1) & 1, abort_flag)) {
            bad = true;
            break;
          }
          ++nuse[g][sl];
        }
        if (bad) break;
        tc_fence_after();
        const int r = q % 3;
        const uint64_t adesc0 = sdesc(sbase + s * kStageZ, kPlaneBytes, kRowBytes);
        const uint64_t bdesc0 = sdesc(wsm + r * 9 * kTapZ, kNZ * 16, 128);
        const uint32_t d = tmem + (uint32_t)(g * 64);
#pragma unroll
        for (int t2 = 0; t2 < 9; ++t2) {
          const uint64_t ad = adesc0 + (uint64_t)(((t2 % 3) * 16 + (t2 / 3) * kRowBytes) >> 4);
          const uint64_t bd = bdesc0 + (uint64_t)((t2 * kTapZ) >> 4);
          umma_bf16(d, ad, bd, idesc, (q == 0 && t2 == 0) ? 0u : 1u);
        }
        umma_commit(EMPTY + 8 * s);                          // the box may be overwritten
        umma_commit(OFULL + 8 * (3 * g + (q + 2) % 3));      // output q - 1 complete
        if (q == L + 1) {                                     // outputs L + 1 and L + 2 (dropped)
          umma_commit(OFULL + 8 * (3 * g + (L + 1) % 3));
          umma_commit(OFULL + 8 * (3 * g + (L + 2) % 3));
        }
        ++j;
      }
      if (bad) {
        atomicCAS(a.err, 0, 2);
        *abort_flag = 1;
      }
      umma_commit(DRAIN);
      if (!mbar_wait(DRAIN, 0, nullptr)) atomicCAS(a.err, 0, 6);
    }
  } else {
    // ---- epilogue: warps 2..5 own TMEM sub-partitions 2, 3, 0, 1 ----
    const int sub = warp & 3;
    const int row = sub * 32 + lane;
    const int xx = row % kTX, yy = row / kTX;
    float bias[kCh];
#pragma unroll
    for (int c = 0; c < kCh; ++c) bias[c] = a.bias[c];
    int nfull[2][3] = {{0, 0, 0}, {0, 0, 0}};
    ZmIter it;
    it.init(blockIdx.x, gridDim.x, nseg, nzs, nz);
    int g, sg, q, L;
    bool stop = false;
    while (!stop && it.next(g, sg, q, L)) {
      const int col = sg / nzs, z0 = (sg % nzs) * kZS;
      const int tx = col % a.ntx, ty = col / a.ntx;
      const int x = tx * kTX + xx, y = ty * kTY + yy;
      // outputs completed by this item: q - 1, and after the last input L + 1 and L + 2
      const int nout = (q == L + 1) ? 3 : 1;
      for (int o = 0; o < nout; ++o) {
        const int u = (o == 0) ? q - 1 : L + o;
        const int sl = (u + 3) % 3;
        bool ok = true;
        if (lane == 0) ok = mbar_wait(OFULL + 8 * (3 * g + sl), nfull[g][sl] & 1, abort_flag);
        ++nfull[g][sl];
        if (!__all_sync(0xffffffffu, ok)) {
          if (lane == 0) {
            atomicCAS(a.err, 0, 3);
            *abort_flag = 1;
          }
          stop = true;
          break;
        }
        tc_fence_after();
        const uint32_t tb = tmem + ((uint32_t)(sub * 32) << 16) + (uint32_t)(g * 64 + sl * kCh);
        const bool real = u >= 1 && u <= L;
        float v[kCh];
        if (real) tmem_ld16(tb, v);
        tmem_zero16(tb);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(OEMPTY + 8 * (3 * g + sl));
        if (real && x < a.nx && y < a.ny) {
          const int z = z0 + u - 1;
          if (MODE == 0) {
            __align__(16) __nv_bfloat16 ov[kCh];
#pragma unroll
            for (int c = 0; c < kCh; ++c) ov[c] = __float2bfloat16(gelu_tc(v[c] + bias[c]));
            const long long p = ((long long)(z + 1) * a.py + (y + 1)) * a.px + (x + 1);
            uint4 *dst = reinterpret_cast<uint4 *>(a.act_out);
            dst[p] = reinterpret_cast<const uint4 *>(ov)[0];
            dst[a.plane + p] = reinterpret_cast<const uint4 *>(ov)[1];
          } else {
            a.out[((long long)z * a.ny + y) * a.nx + x] = v[0] + bias[0];
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(kTmemZ) : "memory");
  }
}

// ---------------------------------------------------------------------------------
// layout helpers
// ---------------------------------------------------------------------------------
// z-march weights: [layer][rotation r][in-plane tap t2 = dx + 3 dy][k chunk][n = 16 slot + co][8 ci].
// Column block `slot` of rotation r feeds the output plane in that slot: with input plane q
// (r = q mod 3) and the slot's output u = q + d (d = (slot - r) mod 3 as -1, 0, +1 ->
// d = 2, 0, 1), the tap's plane offset is p - z = -d, i.e. box plane dz = 1 - (u - q).
__global__ void k_pack_zm(const float *w32, int lstride, __nv_bfloat16 *wpk) {
  const int per_layer = 3 * 9 * 2 * kNZ * 8;
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kNLayers * per_layer) return;
  const int l = e / per_layer;
  int r0 = e - l * per_layer;
  const int ci8 = r0 % 8; r0 /= 8;
  const int n = r0 % kNZ; r0 /= kNZ;
  const int kc = r0 % 2; r0 /= 2;
  const int t2 = r0 % 9; r0 /= 9;
  const int rot = r0;                       // 0..2
  const int slot = n / kCh, co = n % kCh;
  const int d = (slot - rot + 3) % 3;       // 0: u = q, 1: u = q + 1, 2: u = q - 1
  const int dz = d == 0 ? 1 : (d == 1 ? 0 : 2);
  const int tap = t2 + 9 * dz, ci = kc * 8 + ci8;
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
    cuuint32_t box1[4] = {8u * kBX, (cuuint32_t)kBY, 1, 2};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = fn(&p->map1[k], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, p->buf[k], dims, strides, box1, es,
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

size_t conv_packed_elems() { return (size_t)kNLayers * (kWZ / 2); }

int conv_pack_weights(const float *w32, int layer_stride, __nv_bfloat16 *wpk, cudaStream_t s) {
  k_pack_zm<<<(int)((conv_packed_elems() + 255) / 256), 256, 0, s>>>(w32, layer_stride, wpk);
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
  const int nzs = (p->nz + kZS - 1) / kZS;
  const int nseg = a.ntx * a.nty * nzs;
  a.ntiles = nseg;
  a.plane = p->plane;
  a.out = p->out;
  a.err = p->err;
  const int grid = nseg < kCtaPerSm * p->nsm ? nseg : kCtaPerSm * p->nsm;
  MSG_CUDA(cudaFuncSetAttribute(k_conv_zm<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemZ));
  MSG_CUDA(cudaFuncSetAttribute(k_conv_zm<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemZ));
  MSG_CUDA(cudaMemsetAsync(p->err, 0, 4, s));
  int in = 0, nxt = 1;
  for (int l = 0; l < kNLayers; ++l) {
    a.w = wpk + (size_t)l * (kWZ / 2);
    a.bias = bias[l];
    if (l < kNLayers - 1) {
      a.act_out = p->buf[nxt];
      k_conv_zm<0><<<grid, kThreadsTC, kSmemZ, s>>>(p->map1[in], a, nseg, nzs, p->nz);
      MSG_CHECK_LAUNCH();
      a.withhold = -1;
      in = nxt;
      nxt = (nxt == 1) ? 2 : 1;
    } else {
      a.act_out = nullptr;
      k_conv_zm<1><<<grid, kThreadsTC, kSmemZ, s>>>(p->map1[in], a, nseg, nzs, p->nz);
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
