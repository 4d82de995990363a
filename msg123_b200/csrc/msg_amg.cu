// msg_amg.cu -- smoothed-aggregation AMG on the GPU: setup (strength filter, MIS-2
// aggregation, smoothed prolongation, transpose, Galerkin product) and the Jacobi
// V-cycle with a dense FP64 inverse at the coarsest level.
//
// Reference counterparts: make_amgmat / make_grapfilt / make_prolomat /
// trans_prolo2restr / make_galerkin (Make_amg_matrix.f90:20-631) and loop_amg
// (Linear_solution.f90:495-740).  The reference aggregation is a serial max-heap
// (Make_amg_matrix.f90:113-222, :633-768); here it is a deterministic distance-2
// maximal independent set computed in synchronous rounds, so the aggregates do not
// depend on thread scheduling.  Every summation order is fixed (see the Galerkin
// kernel), which makes the whole hierarchy bit-identical to the CPU oracle's.
//
// Level 1 is the context's structured Jacobian (DIA for the V-cycle, its CSR image
// for the setup); levels >= 2 are CSR with the diagonal held apart, as in the
// reference's array_var(level)%{dmat,lumat}.
#include "msg_ctx.cuh"
#include <cooperative_groups.h>
#include <cuda_bf16.h>
#include <vector>
#include <algorithm>

namespace cg = cooperative_groups;

namespace msg {

struct AmgLevel {
  int n = 0, nnz = 0;           // rows, off-diagonal entries
  int *rowptr = nullptr, *col = nullptr;
  double *diag = nullptr, *val = nullptr;
  // transfer to/from the next finer level (held by this, the coarser, level)
  int pnnz = 0;
  int *pptr = nullptr, *pcol = nullptr;   // P: fine rows
  double *pval = nullptr;
  int *rptr = nullptr, *rcol = nullptr;   // R = P^T: coarse rows, fine index ascending
  double *rval = nullptr;
  int *agg = nullptr;                     // aggregate of each fine row (-1: none)
  double *cinv = nullptr;                 // dense inverse (coarsest level only)
  double *x = nullptr, *b = nullptr, *r = nullptr, *x2 = nullptr;
  // mixed precision images
  float *diag_f = nullptr, *val_f = nullptr, *pval_f = nullptr, *rval_f = nullptr;
  __nv_bfloat16 *val_h = nullptr;
  float *xf = nullptr, *bf = nullptr, *rf = nullptr, *x2f = nullptr;
};

struct AmgState {
  std::vector<AmgLevel> lv;
  int *col0 = nullptr;           // level-1 CSR columns, 0-based
  double *val0 = nullptr;        // level-1 CSR values (from the DIA Jacobian)
  int *cnt = nullptr;            // device counter
  int *hcnt = nullptr;           // pinned
  size_t cap_n = 0;              // scratch capacity (rows)
  size_t sflag_cap = 0;
  double *r0 = nullptr, *t0 = nullptr;   // level-1 V-cycle work vectors
  float *x0f = nullptr, *t0f = nullptr, *r0f = nullptr;   // level-1 FP32 work vectors (precision = 1)
  float *b0f = nullptr;                                   // FP32 rounding of the cycle's right-hand side
  // setup scratch
  unsigned char *sflag = nullptr;
  int *has = nullptr, *st = nullptr, *flag = nullptr, *aggid = nullptr, *agg2 = nullptr, *tmpi = nullptr;
  unsigned long long *t0m = nullptr, *t1 = nullptr, *t2 = nullptr;
  double *tdm = nullptr;
  // mixed precision level-1 images
  float *d1f = nullptr, *lu1f = nullptr;
  // Device arena for everything one hierarchy build allocates (levels, transfer operators,
  // Galerkin temporaries): a bump pointer reset at each rebuild, so rebuilds never go to
  // the allocator.  A build that outgrows it takes the rest from the stream-ordered pool
  // and the arena is enlarged before the next build.
  char *arena = nullptr;
  size_t arena_cap = 0, arena_used = 0, arena_spill = 0;
};

static AmgState *S(msg_ctx *c) { return reinterpret_cast<AmgState *>(c->amg); }
static int nb(int n) { return (n + kThreads - 1) / kThreads; }

// ---------------------------------------------------------------------------------
// Strength filter (make_grapfilt, Make_amg_matrix.f90:67-111):
//   strong(i,k) <=> lu_k^2 > |d_i d_j theta^2| and d_i d_j lu_k > 0
//   tdm_i = d_i + sum of the weak lu_k in CSR order
// ---------------------------------------------------------------------------------
__global__ void k_strength(int n, const int *rowptr, const int *col, const double *val, const double *diag,
                           double th2, unsigned char *sflag, int *has, double *tdm) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double di = diag[i], t = di;
  int h = 0;
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    int j = col[k];
    double ddmat = __dmul_rn(di, diag[j]);
    double lu = val[k];
    bool s = (__dmul_rn(lu, lu) > fabs(__dmul_rn(ddmat, th2))) && (__dmul_rn(ddmat, lu) > 0.0);
    sflag[k] = s;
    if (s) h = 1;
    else t = __dadd_rn(t, lu);
  }
  has[i] = h;
  tdm[i] = t;
}

// ---------------------------------------------------------------------------------
// MIS-2 in synchronous rounds.  Tuple = state(2 bits) | hash priority(30) | index(32);
// state 0 = decided non-root or no strong link (never wins), 1 = undecided, 2 = root.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ unsigned mis_hash(unsigned x, unsigned lev) {
  x ^= 0x9e3779b9u * (lev + 1u);
  x ^= x >> 16; x *= 0x7feb352dU; x ^= x >> 15; x *= 0x846ca68bU; x ^= x >> 16;
  return x;
}
__device__ __forceinline__ unsigned long long mis_tuple(int state, int i, int lev) {
  if (state == 0) return 0ull;
  return ((unsigned long long)state << 62) | ((unsigned long long)(mis_hash((unsigned)i, (unsigned)lev) & 0x3fffffffu) << 32) |
         (unsigned long long)(unsigned)i;
}

__global__ void k_mis_init(int n, const int *has, int *st) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) st[i] = has[i] ? 1 : 0;
}

// FROM_STATE: source tuples computed from st; else read from src.
__global__ void k_mis_tuple(int n, const int *st, unsigned long long *t0, int lev) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) t0[i] = mis_tuple(st[i], i, lev);
}

__global__ void k_mis_max(int n, const int *rowptr, const int *col, const unsigned char *sflag,
                          const unsigned long long *src, unsigned long long *dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long m = src[i];
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    if (!sflag[k]) continue;
    unsigned long long v = src[col[k]];
    if (v > m) m = v;
  }
  dst[i] = m;
}

// Decide the undecided nodes of this round and write the next round's tuples (t0); when
// `undecided` is given, count the nodes still undecided (one atomic per warp).
__global__ void k_mis_update(int n, int *st, const unsigned long long *t2, unsigned long long *t0, int lev,
                             int *undecided) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool und = false;
  if (i < n) {
    int s = st[i];
    if (s == 1) {
      unsigned long long t = t2[i];
      if ((unsigned)(t & 0xffffffffull) == (unsigned)i) s = 2;
      else if ((t >> 62) == 2ull) s = 0;
      else und = true;
      st[i] = s;
    }
    t0[i] = mis_tuple(s, i, lev);
  }
  if (undecided) {
    unsigned b = __ballot_sync(0xffffffffu, und);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(undecided, __popc(b));
  }
}

__global__ void k_root_flag(int n, const int *st, int *flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = (st[i] == 2);
}

// pass A: roots keep their id; others join the best root among strong neighbours
__global__ void k_agg_a(int n, const int *rowptr, const int *col, const unsigned char *sflag, const int *st,
                        const int *aggid, int *agg2, int lev) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (st[i] == 2) { agg2[i] = aggid[i]; return; }
  unsigned long long best = 0; int bj = -1;
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    if (!sflag[k]) continue;
    int j = col[k];
    if (st[j] == 2) {
      unsigned long long v = mis_tuple(1, j, lev);
      if (v > best) { best = v; bj = j; }
    }
  }
  agg2[i] = bj >= 0 ? aggid[bj] : -1;
}

// pass B: unassigned rows join the best already-assigned strong neighbour
__global__ void k_agg_b(int n, const int *rowptr, const int *col, const unsigned char *sflag, const int *agg2,
                        int *agg, int lev) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (agg2[i] >= 0) { agg[i] = agg2[i]; return; }
  unsigned long long best = 0; int bj = -1;
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    if (!sflag[k]) continue;
    int j = col[k];
    if (agg2[j] >= 0) {
      unsigned long long v = mis_tuple(1, j, lev);
      if (v > best) { best = v; bj = j; }
    }
  }
  agg[i] = bj >= 0 ? agg2[bj] : -1;
}

// ---------------------------------------------------------------------------------
// Smoothed prolongation (make_prolomat, Make_amg_matrix.f90:224-371):
//   columns in first-appearance order over the strong neighbours (CSR order), then
//   the row's own aggregate; values v = -sum lu over strong j of that aggregate,
//   v = v*omega/tdm, own += 1 - omega.
// ---------------------------------------------------------------------------------
constexpr int kPRowMax = 96;   // longer prolongation rows stop the coarsening (CPU oracle: same rule)
__global__ void k_p_count(int n, const int *rowptr, const int *col, const unsigned char *sflag, const int *agg,
                          int *cnt, int *overflow) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int list[kPRowMax];
  int m = 0;
  bool ovf = false;
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    if (!sflag[k]) continue;
    int J = agg[col[k]];
    if (J < 0) continue;
    bool f = false;
    for (int q = 0; q < m; ++q) if (list[q] == J) { f = true; break; }
    if (!f) { if (m < kPRowMax) list[m++] = J; else ovf = true; }
  }
  int own = agg[i];
  if (own >= 0) {
    bool f = false;
    for (int q = 0; q < m; ++q) if (list[q] == own) { f = true; break; }
    if (!f) { if (m < kPRowMax) list[m++] = own; else ovf = true; }
  }
  if (ovf) atomicExch(overflow, 1);
  cnt[i] = m;
}

__global__ void k_p_fill(int n, const int *rowptr, const int *col, const double *val, const unsigned char *sflag,
                         const int *agg, const double *tdm, double om, const int *pptr, int *pcol, double *pval) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = pptr[i], e = pptr[i + 1];
  int m = 0;
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    if (!sflag[k]) continue;
    int J = agg[col[k]];
    if (J < 0) continue;
    int q;
    for (q = 0; q < m; ++q) if (pcol[b + q] == J) break;
    if (q == m && b + m < e) { pcol[b + m] = J; pval[b + m] = 0.0; m++; }
  }
  int own = agg[i];
  if (own >= 0) {
    int q;
    for (q = 0; q < m; ++q) if (pcol[b + q] == own) break;
    if (q == m && b + m < e) { pcol[b + m] = own; pval[b + m] = 0.0; m++; }
  }
  if (m == 0) return;
  for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) {
    if (!sflag[k]) continue;
    int J = agg[col[k]];
    if (J < 0) continue;
    for (int q = 0; q < m; ++q)
      if (pcol[b + q] == J) { pval[b + q] = __dsub_rn(pval[b + q], val[k]); break; }
  }
  double t = tdm[i];
  for (int q = 0; q < m; ++q) pval[b + q] = __ddiv_rn(__dmul_rn(pval[b + q], om), t);
  if (own >= 0)
    for (int q = 0; q < m; ++q)
      if (pcol[b + q] == own) { pval[b + q] = __dsub_rn(__dadd_rn(pval[b + q], 1.0), om); break; }
}

// R = P^T: counts, atomic fill, then sort every row by fine index (keys are unique).
__global__ void k_r_count(int pnnz, const int *pcol, int *rcnt) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < pnnz) atomicAdd(&rcnt[pcol[q]], 1);
}
__global__ void k_r_fill(int nf, const int *pptr, const int *pcol, const double *pval, const int *rptr, int *fill,
                         int *rcol, double *rval) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  for (int q = pptr[i]; q < pptr[i + 1]; ++q) {
    int J = pcol[q];
    int pos = rptr[J] + atomicAdd(&fill[J], 1);
    rcol[pos] = i;
    rval[pos] = pval[q];
  }
}
// one warp per row; rank sort in shared memory (rows up to 1024 entries, longer rows
// fall back to an in-place insertion sort by lane 0)
constexpr int kRSortCap = 1024;
__global__ void __launch_bounds__(128) k_r_sort(int nc, const int *rptr, int *rcol, double *rval) {
  __shared__ int sc[4][kRSortCap];
  __shared__ double sv[4][kRSortCap];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int row = blockIdx.x * 4 + w;
  if (row >= nc) return;
  int b = rptr[row], m = rptr[row + 1] - b;
  if (m <= 1) return;
  if (m > kRSortCap) {
    if (lane == 0) {
      for (int a = 1; a < m; ++a) {
        int c0 = rcol[b + a]; double v0 = rval[b + a]; int q = a - 1;
        while (q >= 0 && rcol[b + q] > c0) { rcol[b + q + 1] = rcol[b + q]; rval[b + q + 1] = rval[b + q]; --q; }
        rcol[b + q + 1] = c0; rval[b + q + 1] = v0;
      }
    }
    return;
  }
  for (int t = lane; t < m; t += 32) { sc[w][t] = rcol[b + t]; sv[w][t] = rval[b + t]; }
  __syncwarp();
  for (int t = lane; t < m; t += 32) {
    int key = sc[w][t], rank = 0;
    for (int u = 0; u < m; ++u) rank += (sc[w][u] < key);
    rcol[b + rank] = key;
    rval[b + rank] = sv[w][t];
  }
}

// ---------------------------------------------------------------------------------
// Row-wise sparse product C = A*B with deterministic accumulation: A's entries of a
// row are visited in order (its diagonal first when given), and for each of them the
// lanes of a warp add coef*B(j,:) into a per-warp hash table.  B's rows hold unique
// columns, so within one step every table slot receives at most one addition: each
// column is summed in the order of A's entries, the order the CPU oracle uses.
// Output columns ascending; with split_diag the diagonal goes to cdiag (1.0 if absent).
// PASS 0 counts, PASS 1 writes.  Rows with more than kHashMax distinct columns set
// *overflow, and the caller stops coarsening at that level.
// ---------------------------------------------------------------------------------
constexpr int kHash = 1024, kHashMax = 700, kSpgWarps = 3, kPf = 8;
constexpr int kHashSmall = 256, kSmallMaxCols = 120;   // fill-pass table for rows of <= 120 columns

// HASH = table slots per warp.  The fill pass (PASS 1) knows each row's column count from
// the count pass: rows of at most kSmallMaxCols columns go through the kHashSmall variant
// (a quarter of the shared memory, twice the resident warps), the others through kHash.
template <int PASS, int HASH = kHash>
__global__ void __launch_bounds__(32 * kSpgWarps) k_spgemm(int nrows, const int *ap, const int *ac, const double *av,
                                                           const double *adiag, const int *bp, const int *bc,
                                                           const double *bv, int split_diag, int *ocnt,
                                                           const int *cptr, int *ccol, double *cval, double *cdiag,
                                                           int *overflow, const int *rows) {
  constexpr int kComp = (HASH < kHashMax ? HASH : kHashMax) + 32;
  __shared__ int hk[kSpgWarps][HASH];
  __shared__ double hv[kSpgWarps][PASS == 1 ? HASH : 1];
  __shared__ int comp[kSpgWarps][kComp];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int rid = blockIdx.x * kSpgWarps + w;
  if (rid >= nrows) return;
  const int row = rows ? rows[rid] : rid;
  int *K = hk[w];
  double *V = hv[w];
  int a0 = ap[row], a1 = ap[row + 1];
  int start = adiag ? a0 - 1 : a0;
  int m = 0;
  if (PASS == 1) {
    // columns of this row (from the count pass; + 1 for a split-off diagonal)
    m = cptr[row + 1] - cptr[row] + (split_diag ? 1 : 0);
    if ((HASH == kHashSmall) != (m <= kSmallMaxCols)) return;   // the other variant's row
  } else {
    // products of this row -> table size (load factor <= 1/2 when it fits)
    for (int k = start + lane; k < a1; k += 32) {
      int j = (k < a0) ? row : ac[k];
      m += bp[j + 1] - bp[j];
    }
    for (int o = 16; o > 0; o >>= 1) m += __shfl_xor_sync(0xffffffffu, m, o);
  }
  int T = 32;
  while (T < 2 * m && T < HASH) T <<= 1;
  const unsigned mask = (unsigned)T - 1u;
  for (int t = lane; t < T; t += 32) { K[t] = -1; if (PASS == 1) V[t] = 0.0; }
  __syncwarp();
  // PASS 0 only counts distinct columns: no values are loaded, multiplied or added
  auto add = [&](int cc, double p) {
    unsigned hsh = ((unsigned)cc * 2654435761u) & mask;
    for (int probe = 0; probe < T; ++probe) {
      int cur = atomicCAS(&K[hsh], -1, cc);
      if (cur == -1 || cur == cc) {
        if (PASS == 1) V[hsh] = __dadd_rn(V[hsh], p);
        break;
      }
      hsh = (hsh + 1) & mask;
    }
  };
  // kPf entries of A at a time: their B rows (up to 32 entries, one per lane) are loaded
  // together, so the dependent loads of A's column -> B's row bounds -> B's entries overlap
  // across entries; they are then added in entry order exactly as one at a time.
  for (int kb = start; kb < a1; kb += kPf) {
    int cols[kPf], lens[kPf];
    double vals[kPf];
#pragma unroll
    for (int u = 0; u < kPf; ++u) {
      const int k = kb + u;
      lens[u] = 0; cols[u] = -1; vals[u] = 0.0;
      if (k < a1) {
        int j;
        double coef = 0.0;
        if (k < a0) { j = row; if (PASS == 1) coef = adiag[row]; }
        else { j = ac[k]; if (PASS == 1) coef = av[k]; }
        const int b0 = bp[j], len = bp[j + 1] - b0;
        lens[u] = len;
        if (lane < len) {
          cols[u] = bc[b0 + lane];
          if (PASS == 1) vals[u] = __dmul_rn(coef, bv[b0 + lane]);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kPf; ++u) {
      const int k = kb + u;
      if (k < a1) {
        if (lens[u] <= 32) {
          if (lane < lens[u]) add(cols[u], vals[u]);
        } else {   // a B row longer than the warp: the whole row again, in chunks
          int j;
          double coef = 0.0;
          if (k < a0) { j = row; if (PASS == 1) coef = adiag[row]; }
          else { j = ac[k]; if (PASS == 1) coef = av[k]; }
          for (int q = bp[j] + lane; q < bp[j + 1]; q += 32) add(bc[q], PASS == 1 ? __dmul_rn(coef, bv[q]) : 0.0);
        }
      }
      __syncwarp();
    }
  }
  // compact occupied slots
  int u = 0;
  for (int base = 0; base < T; base += 32) {
    int t = base + lane;
    bool occ = K[t] >= 0;
    unsigned bal = __ballot_sync(0xffffffffu, occ);
    if (occ) {
      int pos = u + __popc(bal & ((1u << lane) - 1));
      if (pos < kComp) comp[w][pos] = t;
    }
    u += __popc(bal);
  }
  __syncwarp();
  if (u > kHashMax) {
    if (lane == 0) { atomicExch(overflow, 1); if (PASS == 0) ocnt[row] = 0; }
    return;
  }
  bool hasd = false;
  if (split_diag) {
    for (int t = lane; t < u; t += 32) if (K[comp[w][t]] == row) hasd = true;
    hasd = __any_sync(0xffffffffu, hasd);
  }
  if (PASS == 0) {
    if (lane == 0) ocnt[row] = u - (hasd ? 1 : 0);
    return;
  }
  // rank sort by column
  int out0 = cptr[row];
  if (split_diag && lane == 0) cdiag[row] = 1.0;
  __syncwarp();
  for (int t = lane; t < u; t += 32) {
    int slot = comp[w][t];
    int key = K[slot];
    if (split_diag && key == row) { cdiag[row] = V[slot]; continue; }
    int rank = 0;
    for (int v = 0; v < u; ++v) {
      int k2 = K[comp[w][v]];
      if (split_diag && k2 == row) continue;
      rank += (k2 < key);
    }
    ccol[out0 + rank] = key;
    cval[out0 + rank] = V[slot];
  }
}


// Thread-per-row variant for short rows (at most kTU distinct columns): the products
// are summed one by one in generation order, exactly the CPU oracle's loop.  The column
// set lives in registers (fully unrolled, predicated search, insert and sorting network:
// no dynamically indexed local memory).  Rows that need more columns are appended to
// `longrows` (PASS 0) or skipped (PASS 1) and go through the warp kernel above.
constexpr int kTU = 16, kTM = 64;
template <int PASS>
__global__ void __launch_bounds__(128) k_spgemm_t(int nrows, const int *ap, const int *ac, const double *av,
                                                  const double *adiag, const int *bp, const int *bc, const double *bv,
                                                  int split_diag, int *ocnt, const int *cptr, int *ccol, double *cval,
                                                  double *cdiag, int *longrows, int *nlong) {
  int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= nrows) return;
  int uc[kTU];
  double uv[kTU];
#pragma unroll
  for (int t = 0; t < kTU; ++t) { uc[t] = 0x7fffffff; uv[t] = 0.0; }
  int u = 0;
  int a0 = ap[row], a1 = ap[row + 1];
  int m = 0;
  for (int k = adiag ? a0 - 1 : a0; k < a1; ++k) {
    int j = (k < a0) ? row : ac[k];
    m += bp[j + 1] - bp[j];
  }
  if (m > kTM) {   // long product list: the warp kernel is faster
    if (PASS == 0) longrows[atomicAdd(nlong, 1)] = row;
    return;
  }
  for (int k = adiag ? a0 - 1 : a0; k < a1; ++k) {
    int j = (k < a0) ? row : ac[k];
    double coef = (PASS == 0) ? 0.0 : ((k < a0) ? adiag[row] : av[k]);
    for (int q = bp[j]; q < bp[j + 1]; ++q) {
      int cc = bc[q];
      double p = (PASS == 0) ? 0.0 : __dmul_rn(coef, bv[q]);   // PASS 0 counts columns only
      bool found = false;
#pragma unroll
      for (int t = 0; t < kTU; ++t)
        if (uc[t] == cc) { if (PASS == 1) uv[t] = __dadd_rn(uv[t], p); found = true; }
      if (!found) {
        if (u == kTU) {   // too many columns for the register set
          if (PASS == 0) { longrows[atomicAdd(nlong, 1)] = row; }
          return;
        }
#pragma unroll
        for (int t = 0; t < kTU; ++t)
          if (t == u) { uc[t] = cc; uv[t] = p; }
        ++u;
      }
    }
  }
  if (PASS == 0) {
    int hasd = 0;
    if (split_diag) {
#pragma unroll
      for (int t = 0; t < kTU; ++t) hasd |= (uc[t] == row);
    }
    ocnt[row] = u - hasd;
    return;
  }
  // odd-even transposition sort by column (empty slots hold INT_MAX and stay last)
#pragma unroll
  for (int r = 0; r < kTU; ++r) {
#pragma unroll
    for (int t = r & 1; t + 1 < kTU; t += 2) {
      if (uc[t] > uc[t + 1]) {
        int ci = uc[t]; uc[t] = uc[t + 1]; uc[t + 1] = ci;
        double cv = uv[t]; uv[t] = uv[t + 1]; uv[t + 1] = cv;
      }
    }
  }
  int o = cptr[row];
  if (split_diag) cdiag[row] = 1.0;
#pragma unroll
  for (int t = 0; t < kTU; ++t) {
    if (t < u) {
      if (split_diag && uc[t] == row) { cdiag[row] = uv[t]; continue; }
      ccol[o] = uc[t]; cval[o] = uv[t]; ++o;
    }
  }
}

// ---------------------------------------------------------------------------------
// Dense Gauss-Jordan inverse (partial pivoting, ties to the smallest row), one
// cooperative grid; matrix M is n x 2n row-major in global memory.
// ---------------------------------------------------------------------------------
__global__ void k_dense_fill(int n, const int *rowptr, const int *col, const double *val, const double *diag,
                             double *M) {
  int i = blockIdx.x;
  int w = 2 * n;
  for (int c = threadIdx.x; c < w; c += blockDim.x) M[(size_t)i * w + c] = (c == n + i) ? 1.0 : 0.0;
  __syncthreads();
  if (threadIdx.x == 0) {
    M[(size_t)i * w + i] = diag[i];
    for (int k = rowptr[i]; k < rowptr[i + 1]; ++k) M[(size_t)i * w + col[k]] = val[k];
  }
}

template <bool COOP, int NT>
__global__ void __launch_bounds__(NT) k_gj(int n, double *M, int *piv_out) {
  struct Sync {
    __device__ void operator()() const {
      if (COOP) cg::this_grid().sync();
      else __syncthreads();
    }
  } sync_all;
  __shared__ double sa[NT];
  __shared__ int si[NT];
  const int w = 2 * n;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int p = 0; p < n; ++p) {
    // pivot search by block 0
    if (blockIdx.x == 0) {
      double best = -1.0; int bi = n;
      for (int r = p + threadIdx.x; r < n; r += blockDim.x) {
        double v = fabs(M[(size_t)r * w + p]);
        if (v > best || (v == best && r < bi)) { best = v; bi = r; }
      }
      sa[threadIdx.x] = best; si[threadIdx.x] = bi;
      __syncthreads();
      for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
          double v = sa[threadIdx.x + o]; int r = si[threadIdx.x + o];
          if (v > sa[threadIdx.x] || (v == sa[threadIdx.x] && r < si[threadIdx.x])) { sa[threadIdx.x] = v; si[threadIdx.x] = r; }
        }
        __syncthreads();
      }
      if (threadIdx.x == 0) *piv_out = si[0];
    }
    sync_all();
    int piv = *(volatile int *)piv_out;
    // swap rows p and piv, then scale row p
    if (piv != p)
      for (int c = tid; c < w; c += nth) {
        double t = M[(size_t)p * w + c];
        M[(size_t)p * w + c] = M[(size_t)piv * w + c];
        M[(size_t)piv * w + c] = t;
      }
    sync_all();
    double pinv = __ddiv_rn(1.0, ((volatile double *)M)[(size_t)p * w + p]);
    sync_all();
    for (int c = tid; c < w; c += nth) M[(size_t)p * w + c] = __dmul_rn(M[(size_t)p * w + c], pinv);
    sync_all();
    // eliminate column p from every other row; the factor is read before the row
    // changes (column p included: a_rp - f*a_pp, as the sequential loop computes it)
    {
      const int lane = threadIdx.x & 31;
      const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
      const double *prow = M + (size_t)p * w;
      for (int r = gw; r < n; r += nw) {
        if (r == p) continue;
        double *rrow = M + (size_t)r * w;
        double f = rrow[p];
        __syncwarp();
        if (f == 0.0) continue;
        for (int cc = lane; cc < w; cc += 32) rrow[cc] = __dsub_rn(rrow[cc], __dmul_rn(f, prow[cc]));
        __syncwarp();
      }
    }
    sync_all();
  }
}

// [A | I] from a dense row-major matrix
__global__ void k_dense_fill_rm(int n, const double *a, double *M) {
  int i = blockIdx.x;
  int w = 2 * n;
  for (int c = threadIdx.x; c < w; c += blockDim.x)
    M[(size_t)i * w + c] = (c < n) ? a[(size_t)i * n + c] : ((c == n + i) ? 1.0 : 0.0);
}

__global__ void k_dense_extract(int n, const double *M, double *inv) {
  int i = blockIdx.x;
  for (int j = threadIdx.x; j < n; j += blockDim.x) inv[(size_t)i * n + j] = M[(size_t)i * 2 * n + n + j];
}

// ---------------------------------------------------------------------------------
// V-cycle kernels (loop_amg restated as a Jacobi-smoothed V-cycle)
// ---------------------------------------------------------------------------------
struct Dia {
  int nx, ny, nz, nxy, N;
  const double *d, *lu;
};

__device__ __forceinline__ double dia_row(const Dia &A, int i, const double *x) {
  int iz = i / A.nxy, rem = i - iz * A.nxy, iy = rem / A.nx, ix = rem - iy * A.nx;
  const size_t N = A.N;
  double t = __dmul_rn(A.d[i], x[i]);
  if (iz > 0) t = __dadd_rn(t, __dmul_rn(A.lu[0 * N + i], x[i - A.nxy]));
  if (iy > 0) t = __dadd_rn(t, __dmul_rn(A.lu[1 * N + i], x[i - A.nx]));
  if (ix > 0) t = __dadd_rn(t, __dmul_rn(A.lu[2 * N + i], x[i - 1]));
  if (ix < A.nx - 1) t = __dadd_rn(t, __dmul_rn(A.lu[3 * N + i], x[i + 1]));
  if (iy < A.ny - 1) t = __dadd_rn(t, __dmul_rn(A.lu[4 * N + i], x[i + A.nx]));
  if (iz < A.nz - 1) t = __dadd_rn(t, __dmul_rn(A.lu[5 * N + i], x[i + A.nxy]));
  return t;
}

__device__ __forceinline__ double csr_row(int i, const int *rp, const int *cl, const double *v, const double *d,
                                          const double *x) {
  double t = __dmul_rn(d[i], x[i]);
  for (int k = rp[i]; k < rp[i + 1]; ++k) t = __dadd_rn(t, __dmul_rn(v[k], x[cl[k]]));
  return t;
}

// first sweep from x = 0: r = b exactly, x = 0 + w*b/d
__global__ void k_jac_first(int n, const double *b, const double *d, double w, double *x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = __ddiv_rn(__dmul_rn(w, b[i]), d[i]);
}
__global__ void k_jac_dia(Dia A, const double *b, double w, const double *x, double *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.N; i += gridDim.x * blockDim.x) {
    double r = __dsub_rn(b[i], dia_row(A, i, x));
    y[i] = __dadd_rn(x[i], __ddiv_rn(__dmul_rn(w, r), A.d[i]));
  }
}
__global__ void k_jac_csr(int n, const int *rp, const int *cl, const double *v, const double *d, const double *b,
                          double w, const double *x, double *y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double r = __dsub_rn(b[i], csr_row(i, rp, cl, v, d, x));
    y[i] = __dadd_rn(x[i], __ddiv_rn(__dmul_rn(w, r), d[i]));
  }
}
__global__ void k_res_dia(Dia A, const double *b, const double *x, double *r) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.N; i += gridDim.x * blockDim.x)
    r[i] = __dsub_rn(b[i], dia_row(A, i, x));
}
__global__ void k_res_csr(int n, const int *rp, const int *cl, const double *v, const double *d, const double *b,
                          const double *x, double *r) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    r[i] = __dsub_rn(b[i], csr_row(i, rp, cl, v, d, x));
}
// b_c = R r  (sum in R row order)
__global__ void k_restrict(int nc, const int *rp, const int *rc, const double *rv, const double *r, double *bc) {
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = rp[I]; q < rp[I + 1]; ++q) s = __dadd_rn(s, __dmul_rn(rv[q], r[rc[q]]));
    bc[I] = s;
  }
}
// x += P xc (sum in P row order)
__global__ void k_prolong(int nf, const int *pp, const int *pc, const double *pv, const double *xc, double *x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = pp[i]; q < pp[i + 1]; ++q) s = __dadd_rn(s, __dmul_rn(pv[q], xc[pc[q]]));
    x[i] = __dadd_rn(x[i], s);
  }
}
// x = Cinv b, each row summed in column order
__global__ void k_gemv(int n, const double *Ci, const double *b, double *x) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int j = 0; j < n; ++j) s = __dadd_rn(s, __dmul_rn(Ci[(size_t)i * n + j], b[j]));
  x[i] = s;
}


// ---------------------------------------------------------------------------------
// Mixed-precision V-cycle (precision = 1): FP32 vectors, FP32 level-1 operator and
// transfer weights, BF16 off-diagonals and FP32 diagonal on the coarse levels, FP64
// dense inverse at the coarsest level.  The Krylov recurrences stay FP64: the input r
// is read as double and the output z written as double.
// ---------------------------------------------------------------------------------
struct Dia32 {
  int nx, ny, nz, nxy, N;
  const float *d, *lu;
};


// Row i of the FP32 level-1 operator (DIA: diagonal, then the up, north, west, east, south
// and down off-diagonals) times x, with the cell's grid coordinates given by a 3D launch (x
// from the thread, y from the block's y, the layer from the block's z): no integer
// division per cell.
__device__ __forceinline__ float dia_row3_f(const Dia32 &A, int i, int ix, int iy, int iz, const float *x) {
  const size_t N = A.N;
  float t = A.d[i] * x[i];
  if (iz > 0) t += A.lu[0 * N + i] * x[i - A.nxy];
  if (iy > 0) t += A.lu[1 * N + i] * x[i - A.nx];
  if (ix > 0) t += A.lu[2 * N + i] * x[i - 1];
  if (ix < A.nx - 1) t += A.lu[3 * N + i] * x[i + 1];
  if (iy < A.ny - 1) t += A.lu[4 * N + i] * x[i + A.nx];
  if (iz < A.nz - 1) t += A.lu[5 * N + i] * x[i + A.nxy];
  return t;
}
// Fine-level Jacobi sweep (y = x + w (b - A x) / d) and residual (b - A x) over a 3D grid
// of (32, B/32) thread blocks.
template <typename TY>
__global__ void k_jac_dia3(Dia32 A, const float *__restrict__ b, float w, const float *__restrict__ x, TY *y) {
  const int ix = blockIdx.x * 32 + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y, iz = blockIdx.z;
  if (ix >= A.nx || iy >= A.ny) return;
  const int i = ix + A.nx * (iy + A.ny * iz);
  float r = b[i] - dia_row3_f(A, i, ix, iy, iz, x);
  y[i] = (TY)(x[i] + (w * r) / A.d[i]);
}
__global__ void k_res_dia3(Dia32 A, const float *__restrict__ b, const float *__restrict__ x, float *r) {
  const int ix = blockIdx.x * 32 + threadIdx.x, iy = blockIdx.y * blockDim.y + threadIdx.y, iz = blockIdx.z;
  if (ix >= A.nx || iy >= A.ny) return;
  const int i = ix + A.nx * (iy + A.ny * iz);
  r[i] = b[i] - dia_row3_f(A, i, ix, iy, iz, x);
}

template <typename TB>
__global__ void k_jac_first_f(int n, const TB *b, const float *d, float w, float *x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = (w * (float)b[i]) / d[i];
}
// First fine-level sweep from x = 0; also stores the FP32 rounding of the FP64 right-hand
// side, which every later fine sweep of the cycle reads instead of rounding b again (the
// same values, half the bytes).
// Four elements per thread, all loads issued before the stores: 48 B in flight per thread
// instead of 12, which the one-element form lacked to cover the HBM latency (138 us at
// 25.2M cells, 3.6 TB/s).  Launch with grid4(n, block).
__global__ void k_jac_first_b(int n, const double *__restrict__ b, const float *__restrict__ d, float w,
                              float *__restrict__ x, float *__restrict__ bf) {
  const int st = gridDim.x * blockDim.x;
  for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += 4 * st) {
    double bv[4];
    float dv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * st;
      bv[u] = i < n ? b[i] : 0.0;
      dv[u] = i < n ? d[i] : 1.f;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * st;
      if (i < n) {
        const float bi = (float)bv[u];
        bf[i] = bi;
        x[i] = (w * bi) / dv[u];
      }
    }
  }
}
static int grid4(long long n, int block) { return (int)std::max(1LL, (n + 4LL * block - 1) / (4LL * block)); }
__global__ void k_b2f(int n, const double *b, float *bf) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) bf[i] = (float)b[i];
}
// Coarse levels: four lanes per row (lane q takes entries q, q+4, ... of the row; quad
// shuffle sum).  Each lane issues the column and value loads of four of its entries before
// it gathers x for any of them, and the four gathers before it adds: one memory round trip
// per four entries instead of one per entry (a row of 16 entries is one round trip).  The
// products of a lane are added in entry order.  Every lane reaches the shuffles.
__device__ __forceinline__ float ldf(const float *p) { return *p; }
__device__ __forceinline__ float ldf(const __nv_bfloat16 *p) { return __bfloat162float(*p); }
// Two rows per quad: the quad walks rows 2Q and 2Q+1 together (column and value loads of
// both rows, then the gathers of both), so a warp keeps sixteen rows' loads in flight
// (4% off the mixed V-cycle at 25.2M cells against one row per quad).  Launch with
// grid2r(n): four threads per two rows.
template <typename TV>
__device__ __forceinline__ void csr_off_h4x2(int i0, int q, int n, const int *rp, const int *cl, const TV *v,
                                             const float *x, float &t0, float &t1) {
  float s[2] = {0.f, 0.f};
  int k[2], e[2];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const bool live = i0 + r < n;
    k[r] = live ? rp[i0 + r] + q : 0;
    e[r] = live ? rp[i0 + r + 1] : 0;
  }
  while (k[0] < e[0] || k[1] < e[1]) {
    int c[2][4];
    float a[2][4], xv[2][4];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int kk = k[r] + 4 * u;
        c[r][u] = kk < e[r] ? cl[kk] : -1;
        a[r][u] = kk < e[r] ? ldf(v + kk) : 0.f;
      }
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int u = 0; u < 4; ++u) xv[r][u] = c[r][u] >= 0 ? x[c[r][u]] : 0.f;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (c[r][u] >= 0) s[r] += a[r][u] * xv[r][u];
      k[r] += 16;
    }
  }
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    s[r] += __shfl_xor_sync(0xffffffffu, s[r], 1);
    s[r] += __shfl_xor_sync(0xffffffffu, s[r], 2);
  }
  t0 = s[0];
  t1 = s[1];
}
__global__ void k_jac_csr_h(int n, const int *rp, const int *cl, const __nv_bfloat16 *v, const float *d,
                            const float *b, float w, const float *x, float *y) {
  const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = (int)(gt >> 2) * 2, q = (int)(gt & 3);
  const int i = i0 + (q & 1);        // lanes 0 and 1 of the quad finish rows i0 and i0 + 1
  const bool own = q < 2 && i < n;
  float bi = 0.f, di = 1.f, xi = 0.f;
  if (own) { bi = b[i]; di = d[i]; xi = x[i]; }   // in flight during the row walk
  float o0, o1;
  csr_off_h4x2(i0, q, n, rp, cl, v, x, o0, o1);
  if (own) {
    const float off = q ? o1 : o0;
    const float r = bi - (di * xi + off);
    y[i] = xi + (w * r) / di;
  }
}
__global__ void k_res_csr_h(int n, const int *rp, const int *cl, const __nv_bfloat16 *v, const float *d,
                            const float *b, const float *x, float *r) {
  const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = (int)(gt >> 2) * 2, q = (int)(gt & 3);
  const int i = i0 + (q & 1);
  const bool own = q < 2 && i < n;
  float bi = 0.f, di = 0.f, xi = 0.f;
  if (own) { bi = b[i]; di = d[i]; xi = x[i]; }
  float o0, o1;
  csr_off_h4x2(i0, q, n, rp, cl, v, x, o0, o1);
  if (own) r[i] = bi - (di * xi + (q ? o1 : o0));
}
// 4 threads per two rows
static int grid2r(int n) { return (int)((((long long)n + 1) / 2 * 4 + kThreads - 1) / kThreads); }

// Block-streamed CSR passes of the mixed V-cycle's coarse levels and transfers (the
// CSR-stream scheme of Greathouse and Daga, "Efficient sparse matrix-vector multiplication
// on GPUs using the CSR storage format", SC 2014).  A block owns kSR consecutive rows,
// whose entries are one contiguous range of the CSR arrays: the block walks that range in
// chunks of kSC entries with consecutive threads on consecutive entries (column and value
// loads coalesced, four entries per thread issued before their gathers), parks the
// products in shared memory, and each thread then adds its own row's products in entry
// order.  Rows of any length are handled by the chunk loop.
constexpr int kSR = 128, kSC = 2048, kSU = 4;
enum { kCsrJacobi = 0, kCsrResidual = 1, kCsrRowSum = 2, kCsrAddTo = 3 };
// OP kCsrJacobi: y_i = x_i + w (b_i - d_i x_i - sum_k v_k x_{c_k}) / d_i
// OP kCsrResidual: y_i = b_i - d_i x_i - sum_k v_k x_{c_k}
// OP kCsrRowSum: y_i = sum_k v_k x_{c_k}               (restriction, R = P^T)
// OP kCsrAddTo: y_i = y_i + sum_k v_k x_{c_k}          (prolongation, x += P x_c)
template <int OP, typename TV>
__global__ void __launch_bounds__(kSR) k_csr_stream(int n, const int *__restrict__ rp, const int *__restrict__ cl,
                                                    const TV *__restrict__ v, const float *__restrict__ d,
                                                    const float *__restrict__ b, float w, const float *__restrict__ x,
                                                    float *y) {
  __shared__ float prod[kSC];
  const int t = threadIdx.x;
  const int i0 = blockIdx.x * kSR, i = i0 + t;
  const bool own = i < n;
  const int beg = rp[i0], end = rp[min(i0 + kSR, n)];
  int rb = 0, re = 0;
  float bi = 0.f, di = 1.f, xi = 0.f;
  if (own) {
    rb = rp[i];
    re = rp[i + 1];
    if (OP == kCsrJacobi || OP == kCsrResidual) { bi = b[i]; di = d[i]; xi = x[i]; }
    if (OP == kCsrAddTo) xi = y[i];
  }
  float s = 0.f;
  for (int c0 = beg; c0 < end; c0 += kSC) {
    const int c1 = min(c0 + kSC, end);
    for (int k = c0 + t; k < c1; k += kSR * kSU) {
      int cc[kSU];
      float a[kSU], xv[kSU];
#pragma unroll
      for (int u = 0; u < kSU; ++u) {
        const int kk = k + u * kSR;
        cc[u] = kk < c1 ? cl[kk] : -1;
        a[u] = kk < c1 ? ldf(v + kk) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < kSU; ++u) xv[u] = cc[u] >= 0 ? x[cc[u]] : 0.f;
#pragma unroll
      for (int u = 0; u < kSU; ++u)
        if (cc[u] >= 0) prod[k + u * kSR - c0] = a[u] * xv[u];
    }
    __syncthreads();
    const int lo = max(rb, c0), hi = min(re, c1);
    for (int k = lo; k < hi; ++k) s += prod[k - c0];
    __syncthreads();
  }
  if (!own) return;
  if (OP == kCsrJacobi) y[i] = xi + (w * (bi - (di * xi + s))) / di;
  else if (OP == kCsrResidual) y[i] = bi - (di * xi + s);
  else if (OP == kCsrRowSum) y[i] = s;
  else y[i] = xi + s;
}
static int gridS(int n) { return (n + kSR - 1) / kSR; }
// Restriction b_c = R r: a coarse row gathers from every fine row its aggregate's
// smoothed prolongation reaches (tens of entries), so it is split over four lanes like the
// coarse-level smoother.  Launch with grid2r(nc).
__global__ void k_restrict_f(int nc, const int *rp, const int *rc, const float *rv, const float *r, float *bc) {
  const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int I0 = (int)(gt >> 2) * 2, q = (int)(gt & 3);
  float t0, t1;
  csr_off_h4x2(I0, q, nc, rp, rc, rv, r, t0, t1);
  const int I = I0 + (q & 1);
  if (q < 2 && I < nc) bc[I] = q ? t1 : t0;
}
// Prolongation x += P x_c, a thread per fine row, four rows per thread (rows i0 + u*stride):
// the row bounds, the own values, the first entry of each row and its gather are issued for
// all four rows before any sum (prolongation rows hold 0 to 3 entries, most one or none);
// the rest of a row continues the same in-order sum.  Launch with grid4(nf, block).
__device__ __forceinline__ float csr_row_from(float s, int beg, int end, const int *cl, const float *val,
                                              const float *x) {
  for (int k = beg; k < end; k += 4) {
    int c[4];
    float a[4], xv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int kk = k + u;
      c[u] = kk < end ? cl[kk] : -1;
      a[u] = kk < end ? val[kk] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) xv[u] = c[u] >= 0 ? x[c[u]] : 0.f;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (c[u] >= 0) s += a[u] * xv[u];
  }
  return s;
}
__global__ void k_prolong_f(int nf, const int *__restrict__ pp, const int *__restrict__ pc,
                            const float *__restrict__ pv, const float *__restrict__ xc, float *x) {
  const int st = gridDim.x * blockDim.x;
  for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < nf; i0 += 4 * st) {
    int beg[4], end[4], c[4];
    float a[4], g[4], xi[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * st;
      const bool live = i < nf;
      beg[u] = live ? pp[i] : 0;
      end[u] = live ? pp[i + 1] : 0;
      xi[u] = live ? x[i] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      c[u] = beg[u] < end[u] ? pc[beg[u]] : -1;
      a[u] = beg[u] < end[u] ? pv[beg[u]] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) g[u] = c[u] >= 0 ? xc[c[u]] : 0.f;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * st;
      if (i < nf) {
        float s = 0.f;
        if (c[u] >= 0) s += a[u] * g[u];
        if (beg[u] + 1 < end[u]) s = csr_row_from(s, beg[u] + 1, end[u], pc, pv, xc);
        x[i] = xi[u] + s;
      }
    }
  }
}
// One coarse-level CSR pass.  Measured per pass at 25.2M cells (levels of 2.78M rows x 14
// entries, 204k x 44, 22k x 48, ...): the block-streamed kernel takes 94.6 us per Jacobi
// sweep of the 2.78M-row level against 107.4 for four lanes per row, and 49.6 against 59.4
// for the restriction onto it (5.7 entries per row), but is slower on the short, dense
// levels (28.1 against 24.4 us at 204k rows, 16.1 against 7.8 at 22k) and for the
// prolongation rows (0.6 to 3 entries; 148 against 125 us on the fine grid).  So: long
// levels of short rows stream, the rest runs four lanes per row, prolongation a thread
// per row.
template <int OP, typename TV>
static void csr_pass(int n, int nnz, const int *rp, const int *cl, const TV *v, const float *d, const float *b,
                     float w, const float *x, float *y, cudaStream_t s) {
  const bool stream = OP != kCsrAddTo && n >= (1 << 19) && (long long)nnz <= 24LL * n;
  if (stream) {
    k_csr_stream<OP, TV><<<gridS(n), kSR, 0, s>>>(n, rp, cl, v, d, b, w, x, y);
  } else if constexpr (OP == kCsrJacobi) {
    k_jac_csr_h<<<grid2r(n), kThreads, 0, s>>>(n, rp, cl, v, d, b, w, x, y);
  } else if constexpr (OP == kCsrResidual) {
    k_res_csr_h<<<grid2r(n), kThreads, 0, s>>>(n, rp, cl, v, d, b, x, y);
  } else if constexpr (OP == kCsrRowSum) {
    k_restrict_f<<<grid2r(n), kThreads, 0, s>>>(n, rp, cl, v, x, y);
  } else {
    k_prolong_f<<<grid4(n, kThreads), kThreads, 0, s>>>(n, rp, cl, v, x, y);
  }
}
// coarsest level: FP64 dense inverse applied to a float right-hand side, one warp per
// row (coalesced row reads, fixed shuffle tree).  Launch with n warps; a warp's row index
// is the same in all its lanes, so a warp past the end leaves as a whole.
__global__ void k_gemv_mixed(int n, const double *Ci, const float *b, float *x) {
  const int row = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= n) return;
  double s = 0.0;
  for (int j = lane; j < n; j += 32) s += Ci[(size_t)row * n + j] * (double)b[j];
#pragma unroll
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) x[row] = (float)s;
}
__global__ void k_d2f(int n, const double *a, float *b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (float)a[i];
}
__global__ void k_d2h(int n, const double *a, __nv_bfloat16 *b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = __double2bfloat16(a[i]);
}
__global__ void k_f2d(int n, const float *a, double *b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (double)a[i];
}

__global__ void k_col0(int nnz, const int *offrow1, int *col0) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nnz) col0[k] = offrow1[k] - 1;
}

// ---------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------
// Allocation of one hierarchy build: from the arena, else (arena full) from the pool.
template <typename T>
static int halloc(msg_ctx *c, T **p, size_t n) {
  AmgState *A = S(c);
  const size_t bytes = ((n ? n : 1) * sizeof(T) + 255) & ~(size_t)255;
  if (A->arena && A->arena_used + bytes <= A->arena_cap) {
    *p = reinterpret_cast<T *>(A->arena + A->arena_used);
    A->arena_used += bytes;
    return MSG_OK;
  }
  A->arena_spill += bytes;
  MSG_CUDA(cudaMallocAsync((void **)p, bytes, c->stream));
  return MSG_OK;
}

// Release a pointer from halloc: arena memory is reclaimed at the next reset.
static void hfree(AmgState *A, void *q, cudaStream_t s) {
  if (!q) return;
  const char *b = reinterpret_cast<const char *>(q);
  if (A->arena && b >= A->arena && b < A->arena + A->arena_cap) return;
  cudaFreeAsync(q, s);
}

static void free_level(AmgState *A, AmgLevel &L, cudaStream_t s) {
  void *p[] = {L.rowptr, L.col, L.diag, L.val, L.pptr, L.pcol, L.pval, L.rptr, L.rcol, L.rval, L.agg, L.cinv,
               L.x, L.b, L.r, L.x2, L.diag_f, L.val_f, L.pval_f, L.rval_f, L.val_h, L.xf, L.bf, L.rf, L.x2f};
  for (void *q : p) hfree(A, q, s);
  L = AmgLevel();
}

template <typename T>
static int dalloc(msg_ctx *c, T **p, size_t n) {
  MSG_CUDA(cudaMallocAsync((void **)p, (n ? n : 1) * sizeof(T), c->stream));
  return MSG_OK;
}

static int ensure_scratch(msg_ctx *c, AmgState *A, size_t n, size_t nnz) {
  if (A->cap_n >= n && A->sflag) return MSG_OK;
  cudaStream_t s = c->stream;
  void *p[] = {A->sflag, A->has, A->st, A->flag, A->aggid, A->agg2, A->tmpi, A->t0m, A->t1, A->t2, A->tdm};
  for (void *q : p) if (q) cudaFreeAsync(q, s);
  size_t cn = std::max(n, (size_t)1024);
  int rc;
  A->sflag_cap = std::max(nnz, cn * 7);
  if ((rc = dalloc(c, &A->sflag, A->sflag_cap))) return rc;
  if ((rc = dalloc(c, &A->has, cn))) return rc;
  if ((rc = dalloc(c, &A->st, cn))) return rc;
  if ((rc = dalloc(c, &A->flag, cn))) return rc;
  if ((rc = dalloc(c, &A->aggid, cn))) return rc;
  if ((rc = dalloc(c, &A->agg2, cn))) return rc;
  if ((rc = dalloc(c, &A->tmpi, cn + 1))) return rc;
  if ((rc = dalloc(c, &A->t0m, cn))) return rc;
  if ((rc = dalloc(c, &A->t1, cn))) return rc;
  if ((rc = dalloc(c, &A->t2, cn))) return rc;
  if ((rc = dalloc(c, &A->tdm, cn))) return rc;
  A->cap_n = cn;
  return MSG_OK;
}

static int read_counter(msg_ctx *c, AmgState *A, int *v) {
  MSG_CUDA(cudaMemcpyAsync(A->hcnt, A->cnt, 4, cudaMemcpyDeviceToHost, c->stream));
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  *v = *A->hcnt;
  return MSG_OK;
}


// C = A*B (optionally with A's diagonal first, optionally splitting C's diagonal).
// On return *cptr / *ccol / *cval (and cdiag) are allocated; *ovf set when a row
// exceeds the warp kernel's table, in which case nothing is allocated.
static int spgemm(msg_ctx *c, AmgState *A, int nrows, const int *ap, const int *ac, const double *av,
                  const double *adiag, const int *bp, const int *bc, const double *bv, int split_diag, int **cptr,
                  int **ccol, double **cval, double *cdiag, int *cnnz, int *ovf) {
  cudaStream_t s = c->stream;
  int rc;
  int *cnt = nullptr, *longrows = nullptr, *nl = nullptr;
  *ovf = 0;
  if ((rc = halloc(c, &cnt, nrows + 1))) return rc;
  if ((rc = halloc(c, &longrows, nrows + 1))) return rc;
  if ((rc = halloc(c, &nl, 2))) return rc;
  MSG_CUDA(cudaMemsetAsync(nl, 0, 8, s));
  k_spgemm_t<0><<<(nrows + 127) / 128, 128, 0, s>>>(nrows, ap, ac, av, adiag, bp, bc, bv, split_diag, cnt, nullptr,
                                                   nullptr, nullptr, nullptr, longrows, nl);
  MSG_CHECK_LAUNCH();
  int h[2];
  MSG_CUDA(cudaMemcpyAsync(h, nl, 8, cudaMemcpyDeviceToHost, s));
  MSG_CUDA(cudaStreamSynchronize(s));
  const int nlong = h[0];
  MSG_CUDA(cudaMemsetAsync(A->cnt, 0, 4, s));
  if (nlong > 0) {
    k_spgemm<0><<<(nlong + kSpgWarps - 1) / kSpgWarps, 32 * kSpgWarps, 0, s>>>(
        nlong, ap, ac, av, adiag, bp, bc, bv, split_diag, cnt, nullptr, nullptr, nullptr, nullptr, A->cnt, longrows);
    MSG_CHECK_LAUNCH();
  }
  if ((rc = halloc(c, cptr, nrows + 1))) return rc;
  int tot = 0;
  if ((rc = scan_exclusive(c, cnt, *cptr, nrows, &tot))) return rc;
  if ((rc = read_counter(c, A, ovf))) return rc;
  if (*ovf) {
    hfree(S(c), cnt, s); hfree(S(c), longrows, s); hfree(S(c), nl, s); hfree(S(c), *cptr, s);
    *cptr = nullptr;
    return MSG_OK;
  }
  MSG_CUDA(cudaMemcpyAsync(*cptr + nrows, &tot, 4, cudaMemcpyHostToDevice, s));
  if ((rc = halloc(c, ccol, tot))) return rc;
  if ((rc = halloc(c, cval, tot))) return rc;
  k_spgemm_t<1><<<(nrows + 127) / 128, 128, 0, s>>>(nrows, ap, ac, av, adiag, bp, bc, bv, split_diag, nullptr, *cptr,
                                                   *ccol, *cval, cdiag, nullptr, nullptr);
  MSG_CHECK_LAUNCH();
  if (nlong > 0) {
    k_spgemm<1, kHashSmall><<<(nlong + kSpgWarps - 1) / kSpgWarps, 32 * kSpgWarps, 0, s>>>(
        nlong, ap, ac, av, adiag, bp, bc, bv, split_diag, nullptr, *cptr, *ccol, *cval, cdiag, A->cnt, longrows);
    MSG_CHECK_LAUNCH();
    k_spgemm<1, kHash><<<(nlong + kSpgWarps - 1) / kSpgWarps, 32 * kSpgWarps, 0, s>>>(
        nlong, ap, ac, av, adiag, bp, bc, bv, split_diag, nullptr, *cptr, *ccol, *cval, cdiag, A->cnt, longrows);
    MSG_CHECK_LAUNCH();
  }
  hfree(S(c), cnt, s); hfree(S(c), longrows, s); hfree(S(c), nl, s);
  *cnnz = tot;
  return MSG_OK;
}

// Build level lv+1 from level lv; returns 1 when a coarser level was made, 0 otherwise.
static int coarsen(msg_ctx *c, AmgState *A, int lv, int *made) {
  *made = 0;
  AmgLevel &F = A->lv[lv];
  const int n = F.n;
  int rc;
  if ((rc = ensure_scratch(c, A, n, F.nnz))) return rc;
  if ((size_t)F.nnz > A->sflag_cap) {
    cudaFreeAsync(A->sflag, c->stream);
    if ((rc = dalloc(c, &A->sflag, F.nnz))) return rc;
    A->sflag_cap = F.nnz;
  }
  cudaStream_t s = c->stream;
  double th = (double)c->prm.amg_theta, th2 = th * th;
  k_strength<<<nb(n), kThreads, 0, s>>>(n, F.rowptr, F.col, F.val, F.diag, th2, A->sflag, A->has, A->tdm);
  MSG_CHECK_LAUNCH();
  k_mis_init<<<nb(n), kThreads, 0, s>>>(n, A->has, A->st);
  MSG_CHECK_LAUNCH();
  // t0 = tuples of the current states; t1, t2 = the two max-propagation steps
  unsigned long long *t0 = A->t0m;
  k_mis_tuple<<<nb(n), kThreads, 0, s>>>(n, A->st, t0, lv);
  MSG_CHECK_LAUNCH();
  for (int round = 0; round < 64; ++round) {
    k_mis_max<<<nb(n), kThreads, 0, s>>>(n, F.rowptr, F.col, A->sflag, t0, A->t1);
    MSG_CHECK_LAUNCH();
    k_mis_max<<<nb(n), kThreads, 0, s>>>(n, F.rowptr, F.col, A->sflag, A->t1, A->t2);
    MSG_CHECK_LAUNCH();
    const bool check = (round & 3) == 3 || round == 63;   // a round with nothing undecided is a no-op
    if (check) MSG_CUDA(cudaMemsetAsync(A->cnt, 0, 4, s));
    k_mis_update<<<nb(n), kThreads, 0, s>>>(n, A->st, A->t2, t0, lv, check ? A->cnt : nullptr);
    MSG_CHECK_LAUNCH();
    if (check) {
      int und = 0;
      if ((rc = read_counter(c, A, &und))) return rc;
      if (und == 0) break;
    }
  }
  k_root_flag<<<nb(n), kThreads, 0, s>>>(n, A->st, A->flag);
  MSG_CHECK_LAUNCH();
  int nc = 0;
  if ((rc = scan_exclusive(c, A->flag, A->aggid, n, &nc))) return rc;
  if (nc == 0 || nc >= n) return MSG_OK;
  AmgLevel C;
  C.n = nc;
  if ((rc = halloc(c, &C.agg, n))) return rc;
  k_agg_a<<<nb(n), kThreads, 0, s>>>(n, F.rowptr, F.col, A->sflag, A->st, A->aggid, A->agg2, lv);
  MSG_CHECK_LAUNCH();
  k_agg_b<<<nb(n), kThreads, 0, s>>>(n, F.rowptr, F.col, A->sflag, A->agg2, C.agg, lv);
  MSG_CHECK_LAUNCH();
  // P
  MSG_CUDA(cudaMemsetAsync(A->cnt, 0, 4, s));
  k_p_count<<<nb(n), kThreads, 0, s>>>(n, F.rowptr, F.col, A->sflag, C.agg, A->tmpi, A->cnt);
  MSG_CHECK_LAUNCH();
  {
    int ovp = 0;
    if ((rc = read_counter(c, A, &ovp))) return rc;
    if (ovp) { free_level(A, C, s); return MSG_OK; }
  }
  if ((rc = halloc(c, &C.pptr, n + 1))) return rc;
  int pnnz = 0;
  if ((rc = scan_exclusive(c, A->tmpi, C.pptr, n, &pnnz))) return rc;
  MSG_CUDA(cudaMemcpyAsync(C.pptr + n, &pnnz, 4, cudaMemcpyHostToDevice, s));
  C.pnnz = pnnz;
  if ((rc = halloc(c, &C.pcol, pnnz))) return rc;
  if ((rc = halloc(c, &C.pval, pnnz))) return rc;
  k_p_fill<<<nb(n), kThreads, 0, s>>>(n, F.rowptr, F.col, F.val, A->sflag, C.agg, A->tdm, (double)c->prm.jac_omega,
                                      C.pptr, C.pcol, C.pval);
  MSG_CHECK_LAUNCH();
  // R = P^T
  int *rcnt = nullptr;
  if ((rc = halloc(c, &rcnt, nc + 1))) return rc;
  MSG_CUDA(cudaMemsetAsync(rcnt, 0, (size_t)(nc + 1) * 4, s));
  k_r_count<<<nb(pnnz), kThreads, 0, s>>>(pnnz, C.pcol, rcnt);
  MSG_CHECK_LAUNCH();
  if ((rc = halloc(c, &C.rptr, nc + 1))) return rc;
  int rn = 0;
  if ((rc = scan_exclusive(c, rcnt, C.rptr, nc, &rn))) return rc;
  MSG_CUDA(cudaMemcpyAsync(C.rptr + nc, &rn, 4, cudaMemcpyHostToDevice, s));
  if ((rc = halloc(c, &C.rcol, pnnz))) return rc;
  if ((rc = halloc(c, &C.rval, pnnz))) return rc;
  MSG_CUDA(cudaMemsetAsync(rcnt, 0, (size_t)(nc + 1) * 4, s));
  k_r_fill<<<nb(n), kThreads, 0, s>>>(n, C.pptr, C.pcol, C.pval, C.rptr, rcnt, C.rcol, C.rval);
  MSG_CHECK_LAUNCH();
  k_r_sort<<<(nc + 3) / 4, 128, 0, s>>>(nc, C.rptr, C.rcol, C.rval);
  MSG_CHECK_LAUNCH();
  hfree(A, rcnt, s);
  // AP = A*P (diagonal first)
  int *apptr = nullptr, *apcol = nullptr;
  double *apval = nullptr;
  int apn = 0, ovf = 0;
  if ((rc = spgemm(c, A, n, F.rowptr, F.col, F.val, F.diag, C.pptr, C.pcol, C.pval, 0, &apptr, &apcol, &apval,
                   nullptr, &apn, &ovf)))
    return rc;
  if (ovf) { free_level(A, C, s); return MSG_OK; }
  // A_c = R * AP, diagonal split off
  if ((rc = halloc(c, &C.diag, nc))) return rc;
  int cn = 0;
  if ((rc = spgemm(c, A, nc, C.rptr, C.rcol, C.rval, nullptr, apptr, apcol, apval, 1, &C.rowptr, &C.col, &C.val,
                   C.diag, &cn, &ovf)))
    return rc;
  hfree(A, apptr, s); hfree(A, apcol, s); hfree(A, apval, s);
  if (ovf) { free_level(A, C, s); return MSG_OK; }
  C.nnz = cn;
  if ((rc = halloc(c, &C.x, nc))) return rc;
  if ((rc = halloc(c, &C.b, nc))) return rc;
  if ((rc = halloc(c, &C.r, nc))) return rc;
  if ((rc = halloc(c, &C.x2, nc))) return rc;
  A->lv.push_back(C);
  *made = 1;
  return MSG_OK;
}

static int dense_inverse(msg_ctx *c, AmgLevel &L) {
  int n = L.n, rc;
  cudaStream_t s = c->stream;
  double *M = nullptr;
  int *piv = nullptr;
  if ((rc = halloc(c, &M, (size_t)n * 2 * n))) return rc;
  if ((rc = halloc(c, &piv, 1))) return rc;
  if ((rc = halloc(c, &L.cinv, (size_t)n * n))) return rc;
  k_dense_fill<<<n, 256, 0, s>>>(n, L.rowptr, L.col, L.val, L.diag, M);
  MSG_CHECK_LAUNCH();
  if (n <= 1024) {
    // one block: __syncthreads between the phases of a pivot step
    k_gj<false, 1024><<<1, 1024, 0, s>>>(n, M, piv);
    MSG_CHECK_LAUNCH();
  } else {
    int per_sm = 0, sms = 0;
    MSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gj<true, 256>, 256, 0));
    MSG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    int grid = std::max(1, std::min(sms * std::max(per_sm, 1), (n * 2 * n + 255) / 256));
    void *args[] = {&n, &M, &piv};
    MSG_CUDA(cudaLaunchCooperativeKernel((void *)k_gj<true, 256>, grid, 256, args, 0, s));
    __atomic_fetch_add(&g_launches, 1LL, __ATOMIC_RELAXED);
  }
  k_dense_extract<<<n, 256, 0, s>>>(n, M, L.cinv);
  MSG_CHECK_LAUNCH();
  hfree(S(c), M, s);
  hfree(S(c), piv, s);
  return MSG_OK;
}

void amg_free(msg_ctx *c) {
  AmgState *A = S(c);
  if (!A) return;
  cudaStream_t s = c->stream;
  for (size_t l = 1; l < A->lv.size(); ++l) free_level(A, A->lv[l], s);
  A->lv.clear();
  void *p[] = {A->col0, A->val0, A->cnt, A->r0, A->t0, A->x0f, A->t0f, A->r0f, A->b0f, A->sflag, A->has, A->st, A->flag, A->aggid, A->agg2, A->tmpi, A->t0m, A->t1,
               A->t2, A->tdm, A->d1f, A->lu1f};
  for (void *q : p) if (q) cudaFreeAsync(q, s);
  cudaStreamSynchronize(s);
  if (A->hcnt) cudaFreeHost(A->hcnt);
  if (A->arena) cudaFree(A->arena);
  delete A;
  c->amg = nullptr;
}

// Per-cell bytes of the arena reserved when a context is made: one hierarchy build of the
// block workloads (levels, transfer operators, Galerkin temporaries) takes about 150 B per
// fine cell; a build that outgrows the reservation spills to the pool and the arena is
// enlarged at the next build, as before.
constexpr size_t kArenaPerCell = 192;

static int amg_state(msg_ctx *c);

// Reserve the hierarchy's arena while the context is made, so that the first rebuilds of a
// run allocate nothing: a multi-GB cudaMalloc inside a later rebuild took 50-150 ms more on
// some machines than on others.
int amg_reserve(msg_ctx *c) {
  int rc;
  if ((rc = amg_state(c))) return rc;
  AmgState *A = S(c);
  if (A->arena) return MSG_OK;
  const size_t cap = (kArenaPerCell * (size_t)c->N + ((size_t)1 << 20) - 1) & ~(((size_t)1 << 20) - 1);
  if (cudaMalloc((void **)&A->arena, cap) == cudaSuccess) A->arena_cap = cap;
  else { A->arena = nullptr; A->arena_cap = 0; cudaGetLastError(); }   // the builds use the pool
  // and the setup scratch of the fine level (strength flags, MIS-2 state and tuples,
  // temporaries: about 64 B per cell), which the first build would otherwise take from the
  // pool: at 25.2M cells that first build then cost 20-45 ms more, varying from run to run
  return ensure_scratch(c, A, (size_t)c->N, (size_t)c->nnz);
}

static int amg_state(msg_ctx *c) {
  int rc;
  AmgState *A = S(c);
  cudaStream_t s = c->stream;
  if (!A) {
    A = new AmgState();
    c->amg = A;
    if ((rc = dalloc(c, &A->col0, c->nnz))) return rc;
    if ((rc = dalloc(c, &A->val0, c->nnz))) return rc;
    if ((rc = dalloc(c, &A->cnt, 1))) return rc;
    if ((rc = dalloc(c, &A->r0, c->N))) return rc;
    if ((rc = dalloc(c, &A->t0, c->N))) return rc;
    if (c->prm.precision == 1) {
      if ((rc = dalloc(c, &A->x0f, c->N))) return rc;
      if ((rc = dalloc(c, &A->t0f, c->N))) return rc;
      if ((rc = dalloc(c, &A->r0f, c->N))) return rc;
      if ((rc = dalloc(c, &A->b0f, c->N))) return rc;
    }
    MSG_CUDA(cudaMallocHost((void **)&A->hcnt, 4));
    k_col0<<<nb(c->nnz), kThreads, 0, s>>>(c->nnz, c->offrow, A->col0);
    MSG_CHECK_LAUNCH();
  }
  return MSG_OK;
}

int amg_setup(msg_ctx *c) {
  int rc;
  if ((rc = amg_state(c))) return rc;
  AmgState *A = S(c);
  cudaStream_t s = c->stream;
  for (size_t l = 1; l < A->lv.size(); ++l) free_level(A, A->lv[l], s);
  A->lv.clear();
  // reset the arena; enlarge it first when the previous build did not fit
  if (A->arena_spill) {
    const size_t need = A->arena_used + A->arena_spill;
    if (A->arena) {
      MSG_CUDA(cudaStreamSynchronize(s));
      cudaFree(A->arena);
      A->arena = nullptr;
      A->arena_cap = 0;
    }
    const size_t cap = ((need + need / 4) + ((size_t)1 << 20) - 1) & ~(((size_t)1 << 20) - 1);
    if (cudaMalloc((void **)&A->arena, cap) == cudaSuccess) A->arena_cap = cap;
    else { A->arena = nullptr; cudaGetLastError(); }   // keep using the pool
  }
  A->arena_used = 0;
  A->arena_spill = 0;
  if ((rc = launch_dia_to_csr(c, A->val0))) return rc;
  AmgLevel L0;
  L0.n = c->N; L0.nnz = c->nnz; L0.rowptr = c->offind; L0.col = A->col0; L0.diag = c->dmat; L0.val = A->val0;
  A->lv.push_back(L0);
  int maxlev = std::min(std::max(c->prm.amg_nlevel, 2), 16);
  while ((int)A->lv.size() < maxlev && A->lv.back().n > c->prm.amg_coarse_max) {
    int made = 0;
    if ((rc = coarsen(c, A, (int)A->lv.size() - 1, &made))) return rc;
    if (!made) break;
  }
  if (A->lv.size() > 1 && A->lv.back().n <= std::max(c->prm.amg_coarse_max, 1)) {
    if ((rc = dense_inverse(c, A->lv.back()))) return rc;
  }
  if (c->prm.precision == 1) {
    for (size_t l = 1; l < A->lv.size(); ++l) {
      AmgLevel &L = A->lv[l];
      int nf = A->lv[l - 1].n;
      if ((rc = halloc(c, &L.diag_f, L.n))) return rc;
      if ((rc = halloc(c, &L.val_h, L.nnz))) return rc;
      if ((rc = halloc(c, &L.pval_f, L.pnnz))) return rc;
      if ((rc = halloc(c, &L.rval_f, L.pnnz))) return rc;
      if ((rc = halloc(c, &L.xf, L.n))) return rc;
      if ((rc = halloc(c, &L.bf, L.n))) return rc;
      if ((rc = halloc(c, &L.rf, L.n))) return rc;
      if ((rc = halloc(c, &L.x2f, L.n))) return rc;
      int g = std::min(nb(std::max(L.nnz, L.pnnz)), kRedBlocks * 4);
      k_d2f<<<std::min(nb(L.n), kRedBlocks * 4), kThreads, 0, s>>>(L.n, L.diag, L.diag_f);
      MSG_CHECK_LAUNCH();
      if (L.nnz) { k_d2h<<<g, kThreads, 0, s>>>(L.nnz, L.val, L.val_h); MSG_CHECK_LAUNCH(); }
      k_d2f<<<g, kThreads, 0, s>>>(L.pnnz, L.pval, L.pval_f);
      MSG_CHECK_LAUNCH();
      k_d2f<<<g, kThreads, 0, s>>>(L.pnnz, L.rval, L.rval_f);
      MSG_CHECK_LAUNCH();
      (void)nf;
    }
  }
  c->amg_nlevel = (int)A->lv.size();
  return MSG_OK;
}

// One V-cycle z = M^-1 r (x = 0 start, amg_sweeps Jacobi sweeps before and after).
static int vcycle(msg_ctx *c, int l, const double *b, double *x) {
  AmgState *A = S(c);
  AmgLevel &L = A->lv[l];
  cudaStream_t s = c->stream;
  const int n = L.n, sw = std::max(c->prm.amg_sweeps, 0);
  const double w = (double)c->prm.smooth_omega;
  const int g = nb(n);
  const bool last = (l == (int)A->lv.size() - 1);
  if (last && L.cinv) {
    k_gemv<<<nb(n), kThreads, 0, s>>>(n, L.cinv, b, x);
    MSG_CHECK_LAUNCH();
    return MSG_OK;
  }
  Dia D{c->nx, c->ny, c->nz, c->nxy, c->N, c->dmat, c->lu};
  const int bs = (l == 0 && c->blk_smooth > 0) ? c->blk_smooth : kThreads;
  const int gs = (n + bs - 1) / bs;
  double *r = (l == 0) ? A->r0 : L.r;
  double *tmp = (l == 0) ? A->t0 : L.x2;
  auto sweep = [&](const double *xin, double *xout) {
    if (l == 0) k_jac_dia<<<gs, bs, 0, s>>>(D, b, w, xin, xout);
    else k_jac_csr<<<g, kThreads, 0, s>>>(n, L.rowptr, L.col, L.val, L.diag, b, w, xin, xout);
  };
  // pre-smoothing: the current iterate alternates between x and tmp, so that every
  // sweep reads one buffer and writes the other; total sweeps 2*sw end in x.
  double *cur = x, *oth = tmp;
  if (sw == 0) {
    MSG_CUDA(cudaMemsetAsync(x, 0, (size_t)n * 8, s));
  } else {
    if (sw % 2 == 0) { cur = tmp; oth = x; }
    k_jac_first<<<gs, bs, 0, s>>>(n, b, l == 0 ? c->dmat : L.diag, w, cur);
    MSG_CHECK_LAUNCH();
    for (int k = 1; k < sw; ++k) {
      sweep(cur, oth);
      MSG_CHECK_LAUNCH();
      std::swap(cur, oth);
    }
  }
  if (!last) {
    AmgLevel &C = A->lv[l + 1];
    if (l == 0) k_res_dia<<<gs, bs, 0, s>>>(D, b, cur, r);
    else k_res_csr<<<g, kThreads, 0, s>>>(n, L.rowptr, L.col, L.val, L.diag, b, cur, r);
    MSG_CHECK_LAUNCH();
    k_restrict<<<std::min(nb(C.n), kRedBlocks * 4), kThreads, 0, s>>>(C.n, C.rptr, C.rcol, C.rval, r, C.b);
    MSG_CHECK_LAUNCH();
    int rc = vcycle(c, l + 1, C.b, C.x);
    if (rc) return rc;
    k_prolong<<<gs, bs, 0, s>>>(n, C.pptr, C.pcol, C.pval, C.x, cur);
    MSG_CHECK_LAUNCH();
  }
  for (int k = 0; k < sw; ++k) {
    sweep(cur, oth);
    MSG_CHECK_LAUNCH();
    std::swap(cur, oth);
  }
  if (cur != x) MSG_CUDA(cudaMemcpyAsync(x, cur, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
  return MSG_OK;
}


// Mixed-precision V-cycle on levels >= 1 (float vectors).
static int vcycle_f(msg_ctx *c, int l, const float *b, float *x) {
  AmgState *A = S(c);
  AmgLevel &L = A->lv[l];
  cudaStream_t s = c->stream;
  const int n = L.n, sw = std::max(c->prm.amg_sweeps, 0);
  const float w = c->prm.smooth_omega;
  const int g = nb(n);
  const bool last = (l == (int)A->lv.size() - 1);
  if (last && L.cinv) {
    k_gemv_mixed<<<(int)(((long long)n * 32 + kThreads - 1) / kThreads), kThreads, 0, s>>>(n, L.cinv, b, x);
    MSG_CHECK_LAUNCH();
    return MSG_OK;
  }
  float *cur = x, *oth = L.x2f;
  if (sw == 0) {
    MSG_CUDA(cudaMemsetAsync(x, 0, (size_t)n * 4, s));
  } else {
    if (sw % 2 == 0) { cur = L.x2f; oth = x; }
    k_jac_first_f<float><<<g, kThreads, 0, s>>>(n, b, L.diag_f, w, cur);
    MSG_CHECK_LAUNCH();
    for (int k = 1; k < sw; ++k) {
      csr_pass<kCsrJacobi>(n, L.nnz, L.rowptr, L.col, L.val_h, L.diag_f, b, w, cur, oth, s);
      MSG_CHECK_LAUNCH();
      std::swap(cur, oth);
    }
  }
  if (!last) {
    AmgLevel &C = A->lv[l + 1];
    csr_pass<kCsrResidual>(n, L.nnz, L.rowptr, L.col, L.val_h, L.diag_f, b, 0.f, cur, L.rf, s);
    MSG_CHECK_LAUNCH();
    csr_pass<kCsrRowSum>(C.n, C.pnnz, C.rptr, C.rcol, C.rval_f, nullptr, nullptr, 0.f, L.rf, C.bf, s);
    MSG_CHECK_LAUNCH();
    int rc = vcycle_f(c, l + 1, C.bf, C.xf);
    if (rc) return rc;
    csr_pass<kCsrAddTo>(n, C.pnnz, C.pptr, C.pcol, C.pval_f, nullptr, nullptr, 0.f, C.xf, cur, s);
    MSG_CHECK_LAUNCH();
  }
  for (int k = 0; k < sw; ++k) {
    csr_pass<kCsrJacobi>(n, L.nnz, L.rowptr, L.col, L.val_h, L.diag_f, b, w, cur, oth, s);
    MSG_CHECK_LAUNCH();
    std::swap(cur, oth);
  }
  if (cur != x) MSG_CUDA(cudaMemcpyAsync(x, cur, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
  return MSG_OK;
}

// Level 1 of the mixed V-cycle: r (FP64 Krylov vector) in, z (FP64) out.
static int vcycle_mixed(msg_ctx *c, const double *b, double *z) {
  AmgState *A = S(c);
  cudaStream_t s = c->stream;
  const int n = c->N, sw = std::max(c->prm.amg_sweeps, 0);
  const float w = c->prm.smooth_omega;
  Dia32 D{c->nx, c->ny, c->nz, c->nxy, c->N, c->dmat_f, c->lu_f};
  const bool single = (A->lv.size() == 1);
  const int bs = c->blk_smooth > 0 ? c->blk_smooth : kThreads;
  const int gs = (n + bs - 1) / bs;
  // stencil sweeps: 3D grid, 32 cells of a row per warp, bs / 32 rows per block
  const int by = std::max(bs / 32, 1);
  const dim3 b3(32, by), g3((c->nx + 31) / 32, (c->ny + by - 1) / by, c->nz);
  float *cur = A->x0f, *oth = A->t0f, *bf = A->b0f;
  if (sw == 0) {
    MSG_CUDA(cudaMemsetAsync(cur, 0, (size_t)n * 4, s));
    k_b2f<<<gs, bs, 0, s>>>(n, b, bf);
    MSG_CHECK_LAUNCH();
  } else {
    k_jac_first_b<<<grid4(n, bs), bs, 0, s>>>(n, b, c->dmat_f, w, cur, bf);
    MSG_CHECK_LAUNCH();
    for (int k = 1; k < sw; ++k) {
      k_jac_dia3<float><<<g3, b3, 0, s>>>(D, bf, w, cur, oth);
      MSG_CHECK_LAUNCH();
      std::swap(cur, oth);
    }
  }
  if (!single) {
    AmgLevel &C = A->lv[1];
    k_res_dia3<<<g3, b3, 0, s>>>(D, bf, cur, A->r0f);
    MSG_CHECK_LAUNCH();
    csr_pass<kCsrRowSum>(C.n, C.pnnz, C.rptr, C.rcol, C.rval_f, nullptr, nullptr, 0.f, A->r0f, C.bf, s);
    MSG_CHECK_LAUNCH();
    int rc = vcycle_f(c, 1, C.bf, C.xf);
    if (rc) return rc;
    csr_pass<kCsrAddTo>(n, C.pnnz, C.pptr, C.pcol, C.pval_f, nullptr, nullptr, 0.f, C.xf, cur, s);
    MSG_CHECK_LAUNCH();
  }
  for (int k = 0; k < sw; ++k) {
    if (k == sw - 1) {   // the last sweep writes the FP64 output
      k_jac_dia3<double><<<g3, b3, 0, s>>>(D, bf, w, cur, z);
      MSG_CHECK_LAUNCH();
      return MSG_OK;
    }
    k_jac_dia3<float><<<g3, b3, 0, s>>>(D, bf, w, cur, oth);
    MSG_CHECK_LAUNCH();
    std::swap(cur, oth);
  }
  k_f2d<<<gs, bs, 0, s>>>(n, cur, z);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int amg_apply(msg_ctx *c, const double *r, double *z) {
  if (!S(c) || S(c)->lv.empty()) { set_error("AMG hierarchy not built"); return MSG_ERR_STATE; }
  if (c->prm.precision == 1) return vcycle_mixed(c, r, z);
  return vcycle(c, 0, r, z);
}

}  // namespace msg


// ---------------------------------------------------------------------------------
// Allocation-free dense inverse.
//
// Some callers cannot call cudaMalloc: a Fortran host that hands over device arrays it
// already owns (CUDA Fortran or OpenACC data regions) while its own allocator holds the
// device heap, or a solver step that runs under a fixed device-memory budget where an
// allocation could fail or stall mid-step.  msg_gpu_dense_inverse_noalloc serves them:
// it takes the caller's device buffers and keeps its Gauss-Jordan workspace (the
// augmented [A | I] block and the pivot slot) in the file-scope array below, sized for
// n <= kNoAllocMaxN.  Every GPU that loads this library holds that array (about 4 MiB)
// until the process exits.
// ---------------------------------------------------------------------------------
constexpr int kNoAllocMaxN = 512;
static __device__ __align__(256) double g_noalloc_gj[(size_t)2 * kNoAllocMaxN * kNoAllocMaxN + 32];

// In host code g_noalloc_gj names a host-side stand-in, not device memory: the device
// address comes from cudaGetSymbolAddress with the caller's device current.  It is looked
// up again on every call rather than cached: after a cudaDeviceReset the runtime builds a
// new primary context and reloads this module, and the array may then sit elsewhere, so
// an address kept from before the reset would point into freed memory.  The lookup is a
// host-side table search (the module is loaded by the first call), far cheaper than the
// three kernels it precedes.
static int noalloc_scratch(double **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_gj);
  if (e != cudaSuccess || !p) {
    ::msg::set_error("dense_inverse_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    return MSG_ERR_CUDA;
  }
  *out = static_cast<double *>(p);
  return MSG_OK;
}

// Hierarchy export for structural tests (levels are 0-based; level 0 is the Jacobian).
using namespace msg;
extern "C" {
// Dense FP64 inverse by Gauss-Jordan with partial pivoting: the coarsest-level
// solve of the AMG V-cycle, on host arrays (row-major n x n).
MSG_API int msg_gpu_dense_inverse(int32_t n, const double *a, double *inv) {
  if (n < 1 || !a || !inv) { set_error("dense_inverse: bad arguments"); return MSG_ERR_ARG; }
  double *da = nullptr, *M = nullptr, *dinv = nullptr;
  int *piv = nullptr;
  const size_t nn = (size_t)n * n;
  MSG_CUDA(cudaMalloc(&da, nn * 8));
  MSG_CUDA(cudaMalloc(&M, 2 * nn * 8));
  MSG_CUDA(cudaMalloc(&dinv, nn * 8));
  MSG_CUDA(cudaMalloc(&piv, 4));
  MSG_CUDA(cudaMemcpy(da, a, nn * 8, cudaMemcpyHostToDevice));
  k_dense_fill_rm<<<n, 256>>>(n, da, M);
  MSG_CHECK_LAUNCH();
  if (n <= 1024) {
    k_gj<false, 1024><<<1, 1024>>>(n, M, piv);
    MSG_CHECK_LAUNCH();
  } else {
    int dev = 0, per_sm = 0, sms = 0;
    MSG_CUDA(cudaGetDevice(&dev));
    MSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gj<true, 256>, 256, 0));
    MSG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int grid = std::max(1, std::min(sms * std::max(per_sm, 1), (int)((2 * nn + 255) / 256)));
    int nn32 = n;
    void *args[] = {&nn32, &M, &piv};
    MSG_CUDA(cudaLaunchCooperativeKernel((void *)k_gj<true, 256>, grid, 256, args, 0, 0));
    __atomic_fetch_add(&g_launches, 1LL, __ATOMIC_RELAXED);
  }
  k_dense_extract<<<n, 256>>>(n, M, dinv);
  MSG_CHECK_LAUNCH();
  MSG_CUDA(cudaMemcpy(inv, dinv, nn * 8, cudaMemcpyDeviceToHost));
  cudaFree(da); cudaFree(M); cudaFree(dinv); cudaFree(piv);
  return MSG_OK;
}

// Same result as msg_gpu_dense_inverse, bit for bit, without any allocation: a_dev and
// inv_dev are device arrays (row-major n x n) owned by the caller; the work runs on
// `stream` (NULL: the legacy default stream) and is complete when that stream is.
// Each call looks up the scratch address (cudaGetSymbolAddress) with the current device;
// the first call on a device also loads this module there, so make that first call
// before any stream capture.  All calls share one workspace per device, so calls that
// overlap on the GPU race; each call writes the whole [A | I] block and the pivot slot
// before reading them, so nothing needs to start at zero.  A singular input is not
// detected: a zero pivot gives inf/NaN entries and the call still returns MSG_OK (the
// work is queued, not awaited, so no status can come back from the device).
MSG_API int msg_gpu_dense_inverse_noalloc(int32_t n, const double *a_dev, double *inv_dev, void *stream) {
  if (n < 1 || n > kNoAllocMaxN) {
    set_error("dense_inverse_noalloc: n = %d outside 1..%d (workspace limit)", (int)n, kNoAllocMaxN);
    return MSG_ERR_SIZE;
  }
  if (!a_dev || !inv_dev) { set_error("dense_inverse_noalloc: null device pointer"); return MSG_ERR_ARG; }
  double *M = nullptr;
  int rc = noalloc_scratch(&M);
  if (rc) return rc;
  int *piv = reinterpret_cast<int *>(M + (size_t)2 * kNoAllocMaxN * kNoAllocMaxN);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_dense_fill_rm<<<n, 256, 0, s>>>(n, a_dev, M);
  MSG_CHECK_LAUNCH();
  k_gj<false, 1024><<<1, 1024, 0, s>>>(n, M, piv);
  MSG_CHECK_LAUNCH();
  k_dense_extract<<<n, 256, 0, s>>>(n, M, inv_dev);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

MSG_API int msg_gpu_amg_nlevel(msg_ctx_t *c) {
  return (c && S(c)) ? (int)S(c)->lv.size() : 0;
}
MSG_API int msg_gpu_amg_level_sizes(msg_ctx_t *c, int32_t lv, int32_t *n, int32_t *nnz, int32_t *pnnz) {
  if (!c || !S(c) || lv < 0 || lv >= (int)S(c)->lv.size()) return MSG_ERR_ARG;
  AmgLevel &L = S(c)->lv[lv];
  *n = L.n; *nnz = L.nnz; *pnnz = L.pnnz;
  return MSG_OK;
}
MSG_API int msg_gpu_amg_level(msg_ctx_t *c, int32_t lv, int32_t *offind, int32_t *offrow, double *dmat,
                              double *lumat, int32_t *pindex, int32_t *poffrow, double *pval, int32_t *agg) {
  if (!c || !S(c) || lv < 0 || lv >= (int)S(c)->lv.size()) return MSG_ERR_ARG;
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  AmgLevel &L = S(c)->lv[lv];
  if (offind) MSG_CUDA(cudaMemcpy(offind, L.rowptr, (size_t)(L.n + 1) * 4, cudaMemcpyDeviceToHost));
  if (offrow) MSG_CUDA(cudaMemcpy(offrow, L.col, (size_t)L.nnz * 4, cudaMemcpyDeviceToHost));
  if (dmat) MSG_CUDA(cudaMemcpy(dmat, L.diag, (size_t)L.n * 8, cudaMemcpyDeviceToHost));
  if (lumat) MSG_CUDA(cudaMemcpy(lumat, L.val, (size_t)L.nnz * 8, cudaMemcpyDeviceToHost));
  if (lv > 0) {
    int nf = S(c)->lv[lv - 1].n;
    if (pindex) MSG_CUDA(cudaMemcpy(pindex, L.pptr, (size_t)(nf + 1) * 4, cudaMemcpyDeviceToHost));
    if (poffrow) MSG_CUDA(cudaMemcpy(poffrow, L.pcol, (size_t)L.pnnz * 4, cudaMemcpyDeviceToHost));
    if (pval) MSG_CUDA(cudaMemcpy(pval, L.pval, (size_t)L.pnnz * 8, cudaMemcpyDeviceToHost));
    if (agg) MSG_CUDA(cudaMemcpy(agg, L.agg, (size_t)nf * 4, cudaMemcpyDeviceToHost));
  }
  return MSG_OK;
}
}
