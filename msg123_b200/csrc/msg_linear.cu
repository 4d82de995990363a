// msg_linear.cu -- stencil SpMV, DILU / ILU(0) by hyperplane wavefront, BiCGStab with
// fused dot products, deterministic reductions and scans (B200, sm_100a).
//
// SpMV and the vector updates stream the DIA arrays (d, six off-diagonals) once per
// row: 72 B/row for y = A x in FP64.  One row per thread; reductions write one
// partial per block and a fixed-order second stage (k_finish) sums them, so every
// dot product repeats bit for bit from run to run.
#include "msg_ctx.cuh"
#include <cooperative_groups.h>
#include <vector>
#include <cmath>

namespace cg = cooperative_groups;

namespace msg {

struct Geo3 {
  int nx, ny, nz, nxy, N;
};
static Geo3 geo3(const msg_ctx *c) { return Geo3{c->nx, c->ny, c->nz, c->nxy, c->N}; }
static int nblk(int n) { return (n + kThreads - 1) / kThreads; }

__device__ __forceinline__ void ijk(const Geo3 &g, int i, int &ix, int &iy, int &iz) {
  iz = i / g.nxy;
  int rem = i - iz * g.nxy;
  iy = rem / g.nx;
  ix = rem - iy * g.nx;
}

// ---------------------------------------------------------------------------------
// Exclusive scan of int32 (three phases, 2048 elements per block).
// ---------------------------------------------------------------------------------
constexpr int kScanT = 1024, kScanE = 2048;

__global__ void k_scan_block(const int *in, int *out, int n, int *bsum) {
  __shared__ int s[kScanE];
  int base = blockIdx.x * kScanE;
  for (int t = threadIdx.x; t < kScanE; t += kScanT) s[t] = (base + t < n) ? in[base + t] : 0;
  __syncthreads();
  // Blelloch up-sweep / down-sweep
  int off = 1;
  for (int d = kScanE >> 1; d > 0; d >>= 1) {
    __syncthreads();
    if ((int)threadIdx.x < d) {
      int ai = off * (2 * threadIdx.x + 1) - 1, bi = off * (2 * threadIdx.x + 2) - 1;
      s[bi] += s[ai];
    }
    off <<= 1;
  }
  if (threadIdx.x == 0) { bsum[blockIdx.x] = s[kScanE - 1]; s[kScanE - 1] = 0; }
  for (int d = 1; d < kScanE; d <<= 1) {
    off >>= 1;
    __syncthreads();
    if ((int)threadIdx.x < d) {
      int ai = off * (2 * threadIdx.x + 1) - 1, bi = off * (2 * threadIdx.x + 2) - 1;
      int t = s[ai]; s[ai] = s[bi]; s[bi] += t;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kScanE; t += kScanT)
    if (base + t < n) out[base + t] = s[t];
}

__global__ void k_scan_sums(int *bsum, int nb, int *total) {
  // one thread: nb is at most a few tens of thousands
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int acc = 0;
    for (int b = 0; b < nb; ++b) { int v = bsum[b]; bsum[b] = acc; acc += v; }
    *total = acc;
  }
}

__global__ void k_scan_add(int *out, int n, const int *bsum) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += bsum[i / kScanE];
}

int scan_exclusive(msg_ctx *c, const int *in, int *out, int n, int *total_host) {
  int nb = (n + kScanE - 1) / kScanE;
  int *bsum = nullptr;
  MSG_CUDA(cudaMallocAsync(&bsum, (size_t)(nb + 1) * 4, c->stream));
  k_scan_block<<<nb, kScanT, 0, c->stream>>>(in, out, n, bsum);
  MSG_CHECK_LAUNCH();
  k_scan_sums<<<1, 32, 0, c->stream>>>(bsum, nb, bsum + nb);
  MSG_CHECK_LAUNCH();
  k_scan_add<<<nblk(n), kThreads, 0, c->stream>>>(out, n, bsum);
  MSG_CHECK_LAUNCH();
  if (total_host) {
    MSG_CUDA(cudaMemcpyAsync(total_host, bsum + nb, 4, cudaMemcpyDeviceToHost, c->stream));
    MSG_CUDA(cudaStreamSynchronize(c->stream));
  }
  MSG_CUDA(cudaFreeAsync(bsum, c->stream));
  return MSG_OK;
}

// ---------------------------------------------------------------------------------
// Stencil SpMV y = D x + L/U x in the reference's CSR order (calc_matvec,
// Linear_solution.f90:917-951) and residual r = b - A x (calc_resi,
// Calc_simulation.f90:36-73).  Optional fused dot products into partials:
//   mode 1: (y, w1)            mode 2: (y, w1), (y, y)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ double stencil_row(const Geo3 &g, int i, const double *__restrict__ d,
                                              const double *__restrict__ lu, const double *__restrict__ x) {
  int ix, iy, iz;
  ijk(g, i, ix, iy, iz);
  const size_t N = g.N;
  double t = __dmul_rn(d[i], x[i]);
  if (iz > 0) t = __dadd_rn(t, __dmul_rn(lu[0 * N + i], x[i - g.nxy]));
  if (iy > 0) t = __dadd_rn(t, __dmul_rn(lu[1 * N + i], x[i - g.nx]));
  if (ix > 0) t = __dadd_rn(t, __dmul_rn(lu[2 * N + i], x[i - 1]));
  if (ix < g.nx - 1) t = __dadd_rn(t, __dmul_rn(lu[3 * N + i], x[i + 1]));
  if (iy < g.ny - 1) t = __dadd_rn(t, __dmul_rn(lu[4 * N + i], x[i + g.nx]));
  if (iz < g.nz - 1) t = __dadd_rn(t, __dmul_rn(lu[5 * N + i], x[i + g.nxy]));
  return t;
}

template <int MODE, bool RESID>
__global__ void __launch_bounds__(256) k_spmv(Geo3 g, const double *__restrict__ d, const double *__restrict__ lu,
                                              const double *__restrict__ x, const double *__restrict__ b,
                                              double *__restrict__ y, const double *__restrict__ w1,
                                              double *part) {
  __shared__ double sh[8];
  double a0 = 0.0, a1 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.N; i += gridDim.x * blockDim.x) {
    double t = stencil_row(g, i, d, lu, x);
    if (RESID) t = __dsub_rn(b[i], t);
    y[i] = t;
    if (MODE >= 1) a0 = __dadd_rn(a0, __dmul_rn(t, w1[i]));
    if (MODE >= 2) a1 = __dadd_rn(a1, __dmul_rn(t, t));
  }
  if (MODE >= 1) {
    double s = block_sum<256>(a0, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
  }
  if (MODE >= 2) {
    double s = block_sum<256>(a1, sh);
    if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = s;
  }
}

int launch_spmv(msg_ctx *c, const double *x, double *y) {
  k_spmv<0, false><<<nblk(c->N), 256, 0, c->stream>>>(geo3(c), c->dmat, c->lu, x, nullptr, y, nullptr, nullptr);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

// ---------------------------------------------------------------------------------
// Vector kernels with fused reductions (fixed grid -> deterministic partials).
// ---------------------------------------------------------------------------------
// p = r + beta*(pin - omega*v)  (pin: the previous direction, p itself after the first update)
__global__ void k_bicg_p(int n, const double *pin, double *p, const double *r, const double *v, double beta,
                         double omega) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = __dadd_rn(r[i], __dmul_rn(beta, __dsub_rn(pin[i], __dmul_rn(omega, v[i]))));
}

// x = xin + a*z; r = rin - a*w; partials ||r||^2 and (r, rs).  xin null: x starts at zero
// (0 + a*z, the value the zeroed x gave, without reading it); rin: the residual before the
// update (the right-hand side itself on the first update from x = 0).
__global__ void __launch_bounds__(256) k_bicg_xr(int n, const double *xin, double *x, const double *rin, double *r,
                                                 const double *z, const double *w, const double *rs, double a,
                                                 double *part) {
  __shared__ double sh[8];
  double s0 = 0.0, s1 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = __dadd_rn(xin ? xin[i] : 0.0, __dmul_rn(a, z[i]));
    double ri = __dsub_rn(rin[i], __dmul_rn(a, w[i]));
    r[i] = ri;
    s0 = __dadd_rn(s0, __dmul_rn(ri, ri));
    s1 = __dadd_rn(s1, __dmul_rn(ri, rs[i]));
  }
  double t = block_sum<256>(s0, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
  t = block_sum<256>(s1, sh);
  if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = t;
}

__global__ void __launch_bounds__(256) k_dot2(int n, const double *a, const double *b, const double *cc, double *part) {
  __shared__ double sh[8];
  double s0 = 0.0, s1 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    s0 = __dadd_rn(s0, __dmul_rn(a[i], b[i]));
    if (cc) s1 = __dadd_rn(s1, __dmul_rn(a[i], cc[i]));
  }
  double t = block_sum<256>(s0, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
  if (cc) {
    t = block_sum<256>(s1, sh);
    if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(256) k_norm1(int n, const double *a, double *part) {
  __shared__ double sh[8];
  double s0 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s0 = __dadd_rn(s0, fabs(a[i]));
  double t = block_sum<256>(s0, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_axpby(int n, double *y, const double *x, double a, const double *w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    y[i] = __dadd_rn(x[i], __dmul_rn(a, w[i]));
}

__global__ void k_scale(int n, double *y, double a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = __dmul_rn(y[i], a);
}

// check_abserrmax (Check_simulation.f90:37-91): last index wins ties.
struct ArgMax {
  double a, v;   // |value|, signed value
  int idx;
};
__device__ __forceinline__ ArgMax amax(ArgMax p, ArgMax q) {
  if (q.a > p.a || (q.a == p.a && q.idx > p.idx)) return q;
  return p;
}

// dh non-null: first forms xn = xp + 1*dh (the Newton update, the axpby it replaces, same
// rounding) and writes it, so xn is not read back.
__global__ void __launch_bounds__(256) k_abserrmax(int n, double *xn, const double *xp, const double *dh,
                                                   double *part) {
  __shared__ ArgMax s1[256], s2[256];
  __shared__ int snan[256];
  ArgMax c = {0.0, 0.0, -1}, x = {0.0, 0.0, -1};
  int nan = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v;
    if (dh) {
      v = __dadd_rn(xp[i], __dmul_rn(1.0, dh[i]));
      xn[i] = v;
    } else {
      v = xn[i];
    }
    if (v != v) nan = 1;
    double dv = __dsub_rn(v, xp[i]);
    c = amax(c, ArgMax{fabs(dv), dv, i});
    x = amax(x, ArgMax{fabs(v), v, i});
  }
  s1[threadIdx.x] = c; s2[threadIdx.x] = x; snan[threadIdx.x] = nan;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s1[threadIdx.x] = amax(s1[threadIdx.x], s1[threadIdx.x + o]);
      s2[threadIdx.x] = amax(s2[threadIdx.x], s2[threadIdx.x + o]);
      snan[threadIdx.x] |= snan[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double *q = part + (size_t)blockIdx.x * 8;
    q[0] = s1[0].a; q[1] = s1[0].v; q[2] = (double)s1[0].idx;
    q[3] = s2[0].a; q[4] = s2[0].v; q[5] = (double)s2[0].idx;
    q[6] = (double)snan[0];
  }
}

// lam_length of run_backtr (Nonlinear_solution.f90:503-512): max(1, max_i |dh_i| / |h_i|) over
// h_i != 0.  Rounding is monotone, so the largest rounded quotient is the rounding of the
// largest exact one: each thread keeps the (numerator, denominator) pair of its largest
// exact ratio, comparing a/b with c/d through a*d against c*b exactly (the rounded product
// and its FMA error term), and divides once at the end -- the same value as dividing every
// element, without an FP64 division per cell.
__device__ __forceinline__ bool ratio_greater(double a, double b, double c, double d) {
  const double p1 = a * d, p2 = c * b;
  if (p1 != p2) return p1 > p2;
  return fma(a, d, -p1) > fma(c, b, -p2);
}
__global__ void __launch_bounds__(256) k_lamlen(int n, const double *dh, const double *hn, double *part) {
  __shared__ double s[256];
  double num = 1.0, den = 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double h = fabs(hn[i]), a = fabs(dh[i]);
    if (h != 0.0 && ratio_greater(a, h, num, den)) { num = a; den = h; }
  }
  const double m = __ddiv_rn(num, den);
  s[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

static int fetch_partials(msg_ctx *c, int count) {
  MSG_CUDA(cudaMemcpyAsync(c->hpin, c->part, (size_t)count * 8, cudaMemcpyDeviceToHost, c->stream));
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  return MSG_OK;
}

// Second reduction stage: block a sums part[a*nparts .. a*nparts + nparts) in a fixed
// order, so every result repeats bit for bit: each thread keeps eight running sums over
// the strided elements (eight loads in flight instead of one dependent chain), combines
// them in a fixed tree, then the block reduces in a fixed tree.
// MAXB: bit a set -> block a takes the maximum of its array instead of the sum.
template <int MAXB = 0>
__global__ void __launch_bounds__(1024) k_finish(const double *part, int nparts, double *out) {
  __shared__ double sh[1024];
  const double *p = part + (size_t)blockIdx.x * nparts;
  const bool mx = (MAXB >> blockIdx.x) & 1;
  constexpr int U = 8;
  double a[U];
#pragma unroll
  for (int u = 0; u < U; ++u) a[u] = 0.0;
  for (int base = threadIdx.x; base < nparts; base += U * blockDim.x) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = base + u * blockDim.x;
      if (i < nparts) a[u] = mx ? fmax(a[u], p[i]) : __dadd_rn(a[u], p[i]);
    }
  }
  double s;
  if (mx) s = fmax(fmax(fmax(a[0], a[1]), fmax(a[2], a[3])), fmax(fmax(a[4], a[5]), fmax(a[6], a[7])));
  else s = __dadd_rn(__dadd_rn(__dadd_rn(a[0], a[1]), __dadd_rn(a[2], a[3])),
                     __dadd_rn(__dadd_rn(a[4], a[5]), __dadd_rn(a[6], a[7])));
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      sh[threadIdx.x] = mx ? fmax(sh[threadIdx.x], sh[threadIdx.x + o]) : __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// Second stage into dres[slot .. slot + narr) without waiting: results of several
// reductions come back with one fetch_res (one host round trip).
int finish_to(msg_ctx *c, int nparts, int narr, int slot) {
  k_finish<<<narr, 1024, 0, c->stream>>>(c->part, nparts, c->dres + slot);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int fetch_res(msg_ctx *c, int count, double *out) {
  MSG_CUDA(cudaMemcpyAsync(c->hpin, c->dres, (size_t)count * 8, cudaMemcpyDeviceToHost, c->stream));
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  for (int a = 0; a < count; ++a) out[a] = c->hpin[a];
  return MSG_OK;
}

int finish(msg_ctx *c, int nparts, int narr, double *out) {
  int rc = finish_to(c, nparts, narr, 0);
  if (rc) return rc;
  return fetch_res(c, narr, out);
}

int dot(msg_ctx *c, const double *a, const double *b, int n, double *out) {
  k_dot2<<<nblk(n), 256, 0, c->stream>>>(n, a, b, nullptr, c->part);
  MSG_CHECK_LAUNCH();
  return finish(c, nblk(n), 1, out);
}

int norm1(msg_ctx *c, const double *a, int n, double *out) {
  k_norm1<<<nblk(n), 256, 0, c->stream>>>(n, a, c->part);
  MSG_CHECK_LAUNCH();
  return finish(c, nblk(n), 1, out);
}

int abserrmax(msg_ctx *c, double *xn, const double *xp, double *chmax, double *xmax, int *nun, int *nan,
              const double *dh) {
  k_abserrmax<<<kRedBlocks, 256, 0, c->stream>>>(c->N, xn, xp, dh, c->part);
  MSG_CHECK_LAUNCH();
  int rc = fetch_partials(c, kRedBlocks * 8);
  if (rc) return rc;
  double ca = 0.0, cv = 0.0, xa = 0.0, xv = 0.0;
  long ci = -1, xi = -1;
  int nn = 0;
  for (int b = 0; b < kRedBlocks; ++b) {
    const double *q = c->hpin + (size_t)b * 8;
    long i1 = (long)q[2], i2 = (long)q[5];
    if (i1 >= 0 && (q[0] > ca || (q[0] == ca && i1 > ci))) { ca = q[0]; cv = q[1]; ci = i1; }
    if (i2 >= 0 && (q[3] > xa || (q[3] == xa && i2 > xi))) { xa = q[3]; xv = q[4]; xi = i2; }
    nn |= (int)q[6];
  }
  *nan = nn;
  if (!nn) { *chmax = cv; *xmax = xv; *nun = (int)ci + 1; }
  else { *chmax = 0.0; *xmax = NAN; *nun = 0; }
  return MSG_OK;
}

// The line search's four reductions over the full step in one pass (run_backtr,
// Nonlinear_solution.f90:441-512): ||dh||^2, ||F(h + dh)||^2, the slope (s, J dh) and
// lam_length's largest ratio |dh| / |h|.  The sums use the grid and order of k_dot2, so each
// has the bits of its own dot product; J dh is jv, or b - r (BiCGStab's residual from dh = 0)
// formed with the rounding of the axpby it replaces.  The maximum is exact whatever the grid.
__global__ void __launch_bounds__(256) k_backtr_stats(int n, const double *dh, const double *hn, const double *f,
                                                      const double *s, const double *jv, const double *b,
                                                      const double *r, double *part) {
  __shared__ double sh[8];
  __shared__ double sm[256];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, num = 1.0, den = 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double d = dh[i], fi = f[i];
    s0 = __dadd_rn(s0, __dmul_rn(d, d));
    s1 = __dadd_rn(s1, __dmul_rn(fi, fi));
    const double j = jv ? jv[i] : __dadd_rn(b[i], __dmul_rn(-1.0, r[i]));
    s2 = __dadd_rn(s2, __dmul_rn(s[i], j));
    const double h = fabs(hn[i]), a = fabs(d);
    if (h != 0.0 && ratio_greater(a, h, num, den)) { num = a; den = h; }
  }
  double t = block_sum<256>(s0, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
  t = block_sum<256>(s1, sh);
  if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = t;
  t = block_sum<256>(s2, sh);
  if (threadIdx.x == 0) part[2 * gridDim.x + blockIdx.x] = t;
  sm[threadIdx.x] = __ddiv_rn(num, den);
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[3 * gridDim.x + blockIdx.x] = sm[0];
}

int backtr_stats(msg_ctx *c, const double *dh, const double *hn, const double *f, const double *s, const double *jv,
                 const double *b, const double *r, double out[5], bool slot4) {
  const int nb = nblk(c->N);
  if ((size_t)4 * nb > c->npart) { set_error("backtr_stats: partials buffer too small"); return MSG_ERR_STATE; }
  k_backtr_stats<<<nb, 256, 0, c->stream>>>(c->N, dh, hn, f, s, jv, b, r, c->part);
  MSG_CHECK_LAUNCH();
  k_finish<8><<<4, 1024, 0, c->stream>>>(c->part, nb, c->dres);
  MSG_CHECK_LAUNCH();
  int rc = fetch_res(c, slot4 ? 5 : 4, out);
  if (rc) return rc;
  out[3] = std::fmax(1.0, out[3]);
  return MSG_OK;
}

int lam_length(msg_ctx *c, const double *dh, const double *hn, double *out) {
  k_lamlen<<<kRedBlocks, 256, 0, c->stream>>>(c->N, dh, hn, c->part);
  MSG_CHECK_LAUNCH();
  int rc = fetch_partials(c, kRedBlocks);
  if (rc) return rc;
  double m = 1.0;
  for (int b = 0; b < kRedBlocks; ++b) m = std::fmax(m, c->hpin[b]);
  *out = m;
  return MSG_OK;
}

int axpby(msg_ctx *c, double *y, const double *x, double a, const double *w, int n) {
  k_axpby<<<nblk(n), 256, 0, c->stream>>>(n, y, x, a, w);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int scale(msg_ctx *c, double *y, double a, int n) {
  k_scale<<<nblk(n), 256, 0, c->stream>>>(n, y, a);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

// ---------------------------------------------------------------------------------
// DILU / ILU(0) by hyperplane wavefront.  In natural order on the 7-point stencil
// the lower neighbours of cell (ix,iy,iz) are (ix-1,..), (..,iy-1,..), (..,iz-1), so
// every cell of the plane ix+iy+iz = p depends only on plane p-1: processing planes
// in order, cells of one plane in parallel, performs exactly the sequential
// arithmetic of precon_dilu / solve_ilu (Linear_solution.f90:742-782, :803-855).
// ---------------------------------------------------------------------------------
int build_wavefront(msg_ctx *c) {
  int nx = c->nx, ny = c->ny, nz = c->nz;
  int np = nx + ny + nz - 2;
  std::vector<int> ptr(np + 1, 0), cells(c->N);
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) ptr[ix + iy + iz + 1]++;
  for (int p = 0; p < np; ++p) ptr[p + 1] += ptr[p];
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) cells[fill[ix + iy + iz]++] = ix + nx * (iy + ny * iz);
  c->nplanes = np;
  MSG_CUDA(cudaMalloc(&c->plane_ptr, (size_t)(np + 1) * 4));
  MSG_CUDA(cudaMalloc(&c->plane_cells, (size_t)c->N * 4));
  MSG_CUDA(cudaMemcpy(c->plane_ptr, ptr.data(), (size_t)(np + 1) * 4, cudaMemcpyHostToDevice));
  MSG_CUDA(cudaMemcpy(c->plane_cells, cells.data(), (size_t)c->N * 4, cudaMemcpyHostToDevice));
  return MSG_OK;
}

struct WaveArgs {
  Geo3 g;
  const int *ptr, *cells;
  int nplanes;
  const double *dmat, *lu;
  double *dd;            // DILU diagonal (out for factor, in for solve)
  const double *b;
  double *x;
};

__device__ __forceinline__ void dilu_row(const WaveArgs &a, int i) {
  int ix, iy, iz;
  ijk(a.g, i, ix, iy, iz);
  const size_t N = a.g.N;
  double d = a.dmat[i];
  if (iz > 0) { int j = i - a.g.nxy; double dinv = __ddiv_rn(1.0, a.dd[j]); d = __dsub_rn(d, __dmul_rn(__dmul_rn(a.lu[0 * N + i], dinv), a.lu[5 * N + j])); }
  if (iy > 0) { int j = i - a.g.nx;  double dinv = __ddiv_rn(1.0, a.dd[j]); d = __dsub_rn(d, __dmul_rn(__dmul_rn(a.lu[1 * N + i], dinv), a.lu[4 * N + j])); }
  if (ix > 0) { int j = i - 1;       double dinv = __ddiv_rn(1.0, a.dd[j]); d = __dsub_rn(d, __dmul_rn(__dmul_rn(a.lu[2 * N + i], dinv), a.lu[3 * N + j])); }
  a.dd[i] = d;
}

__device__ __forceinline__ void fwd_row(const WaveArgs &a, int i) {
  int ix, iy, iz;
  ijk(a.g, i, ix, iy, iz);
  const size_t N = a.g.N;
  double t = a.b[i];
  if (iz > 0) t = __dsub_rn(t, __dmul_rn(a.lu[0 * N + i], a.x[i - a.g.nxy]));
  if (iy > 0) t = __dsub_rn(t, __dmul_rn(a.lu[1 * N + i], a.x[i - a.g.nx]));
  if (ix > 0) t = __dsub_rn(t, __dmul_rn(a.lu[2 * N + i], a.x[i - 1]));
  a.x[i] = __ddiv_rn(t, a.dd[i]);
}

__device__ __forceinline__ void bwd_row(const WaveArgs &a, int i) {
  int ix, iy, iz;
  ijk(a.g, i, ix, iy, iz);
  const size_t N = a.g.N;
  double t = 0.0;
  if (ix < a.g.nx - 1) t = __dadd_rn(t, __dmul_rn(a.lu[3 * N + i], a.x[i + 1]));
  if (iy < a.g.ny - 1) t = __dadd_rn(t, __dmul_rn(a.lu[4 * N + i], a.x[i + a.g.nx]));
  if (iz < a.g.nz - 1) t = __dadd_rn(t, __dmul_rn(a.lu[5 * N + i], a.x[i + a.g.nxy]));
  a.x[i] = __dsub_rn(a.x[i], __ddiv_rn(t, a.dd[i]));
}

// MODE 0: factor; MODE 1: forward + backward solve.  COOP: grid-wide sync between
// planes (cooperative launch); otherwise a single block with __syncthreads.
template <int MODE, bool COOP>
__global__ void __launch_bounds__(1024) k_wave(WaveArgs a) {
  auto sync = [&]() {
    if (COOP) cg::this_grid().sync();
    else __syncthreads();
  };
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int p = 0; p < a.nplanes; ++p) {
    int b = a.ptr[p], e = a.ptr[p + 1];
    for (int q = b + tid; q < e; q += nth) {
      if (MODE == 0) dilu_row(a, a.cells[q]);
      else fwd_row(a, a.cells[q]);
    }
    sync();
  }
  if (MODE == 1) {
    for (int p = a.nplanes - 1; p >= 0; --p) {
      int b = a.ptr[p], e = a.ptr[p + 1];
      for (int q = b + tid; q < e; q += nth) bwd_row(a, a.cells[q]);
      sync();
    }
  }
}

static int launch_wave(msg_ctx *c, WaveArgs &a, int mode) {
  const int kSmall = 1 << 18;
  if (c->N <= kSmall) {
    if (mode == 0) k_wave<0, false><<<1, 1024, 0, c->stream>>>(a);
    else k_wave<1, false><<<1, 1024, 0, c->stream>>>(a);
    MSG_CHECK_LAUNCH();
    return MSG_OK;
  }
  int per_sm = 0;
  void *fn = mode == 0 ? (void *)k_wave<0, true> : (void *)k_wave<1, true>;
  MSG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 1024, 0));
  int sms = 0;
  MSG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
  int grid = sms * (per_sm > 0 ? per_sm : 1);
  void *args[] = {&a};
  MSG_CUDA(cudaLaunchCooperativeKernel(fn, grid, 1024, args, 0, c->stream));
  __atomic_fetch_add(&g_launches, 1LL, __ATOMIC_RELAXED);
  return MSG_OK;
}

int launch_precon_dilu(msg_ctx *c) {
  WaveArgs a{geo3(c), c->plane_ptr, c->plane_cells, c->nplanes, c->dmat, c->lu, c->dilu_d, nullptr, nullptr};
  return launch_wave(c, a, 0);
}

int launch_solve_ilu(msg_ctx *c, const double *b, double *x) {
  WaveArgs a{geo3(c), c->plane_ptr, c->plane_cells, c->nplanes, c->dmat, c->lu, c->dilu_d, b, x};
  return launch_wave(c, a, 1);
}

int apply_prec(msg_ctx *c, const double *r, double *z) {
  if (c->prm.precon_type == 0) return launch_solve_ilu(c, r, z);
  if (c->prm.ref_quirks) {
    // loop_amg of the reference returns solve_ilu at level 1 (quirk Q1) and leaves its
    // input in array_var(1)%rhs, which the line-search slope then reads (quirk Q2).
    int rc = launch_solve_ilu(c, r, z);
    if (rc) return rc;
    MSG_CUDA(cudaMemcpyAsync(c->slope_rhs, r, (size_t)c->N * 8, cudaMemcpyDeviceToDevice, c->stream));
    return MSG_OK;
  }
  return amg_apply(c, r, z);
}

// ---------------------------------------------------------------------------------
// solve_bicgs (Linear_solution.f90:234-493): right-preconditioned BiCGStab, x0 = x.
// ---------------------------------------------------------------------------------
int solve_bicgs(msg_ctx *c, double *x, bool x_zero) {
  const int n = c->N;
  const Geo3 g = geo3(c);
  int rc;
  const int nb = nblk(n);
  double red[2];
  double sk = 0.0, sk0 = 1.0e20, sk2, alpha = 0.0, beta, omega = 1.0, ts, tt;
  bool need_dilu = (c->prm.precon_type == 0) || c->prm.ref_quirks;
  // r* (fixed during the solve), the first search direction and the residual before the
  // first update.  From x = 0 all three are b itself: nothing is copied, and x is first
  // written (not read) by the first update.
  const double *rs, *p1, *r1;
  if (x_zero) {
    if (need_dilu && (rc = launch_precon_dilu(c))) return rc;
    // sk = <b, b>, collected with the first (v, r*) in one host round trip
    k_dot2<<<nb, 256, 0, c->stream>>>(n, c->rhs, c->rhs, nullptr, c->part);
    MSG_CHECK_LAUNCH();
    if ((rc = finish_to(c, nb, 1, 2))) return rc;
    rs = p1 = r1 = c->rhs;
  } else {
    // r = b - A x
    k_spmv<0, true><<<nb, 256, 0, c->stream>>>(g, c->dmat, c->lu, x, c->rhs, c->r, nullptr, nullptr);
    MSG_CHECK_LAUNCH();
    if (need_dilu && (rc = launch_precon_dilu(c))) return rc;
    MSG_CUDA(cudaMemcpyAsync(c->rs, c->r, (size_t)n * 8, cudaMemcpyDeviceToDevice, c->stream));
    if ((rc = dot(c, c->r, c->rs, n, &sk))) return rc;
    rs = p1 = c->rs;
    r1 = c->r;
  }
  c->conv_flag = 0;
  for (c->in_iter = 1; c->in_iter <= c->prm.maxinn_iter; ++c->in_iter) {
    const double *p = c->p;
    if (c->in_iter == 1) {
      p = p1;
    } else {
      beta = (sk / sk0) * (alpha / omega);
      k_bicg_p<<<nb, 256, 0, c->stream>>>(n, c->in_iter == 2 ? p1 : c->p, c->p, c->r, c->v, beta, omega);
      MSG_CHECK_LAUNCH();
    }
    if ((rc = apply_prec(c, p, c->z))) return rc;
    k_spmv<1, false><<<nb, 256, 0, c->stream>>>(g, c->dmat, c->lu, c->z, nullptr, c->v, rs, c->part);
    MSG_CHECK_LAUNCH();
    if (x_zero && c->in_iter == 1) {
      double got[3];
      if ((rc = finish_to(c, nb, 1, 0)) || (rc = fetch_res(c, 3, got))) return rc;
      red[0] = got[0];
      sk = got[2];
    } else if ((rc = finish(c, nb, 1, red))) {
      return rc;
    }
    sk2 = red[0];
    alpha = sk / sk2;
    const bool first = (c->in_iter == 1);
    k_bicg_xr<<<nb, 256, 0, c->stream>>>(n, first && x_zero ? nullptr : x, x, first ? r1 : c->r, c->r, c->z, c->v,
                                        rs, alpha, c->part);
    MSG_CHECK_LAUNCH();
    if ((rc = finish(c, nb, 1, red))) return rc;
    c->rnorm = red[0];
    c->conv_flag = (std::sqrt(c->rnorm / c->bnorm) <= c->errtol) ? 1 : 0;
    if (c->conv_flag == 1) break;
    if ((rc = apply_prec(c, c->r, c->z))) return rc;
    k_spmv<2, false><<<nb, 256, 0, c->stream>>>(g, c->dmat, c->lu, c->z, nullptr, c->t, c->r, c->part);
    MSG_CHECK_LAUNCH();
    if ((rc = finish(c, nb, 2, red))) return rc;
    ts = red[0];
    tt = red[1];
    omega = ts / tt;
    k_bicg_xr<<<nb, 256, 0, c->stream>>>(n, x, x, c->r, c->r, c->z, c->t, rs, omega, c->part);
    MSG_CHECK_LAUNCH();
    if ((rc = finish(c, nb, 2, red))) return rc;
    c->rnorm = red[0];
    double sk_next = red[1];
    c->conv_flag = (std::sqrt(c->rnorm / c->bnorm) <= c->errtol) ? 1 : 0;
    if (c->conv_flag == 1 || c->in_iter == c->prm.maxinn_iter) break;
    sk0 = sk;
    sk = sk_next;
  }
  if (c->in_iter > c->prm.maxinn_iter) c->in_iter = c->prm.maxinn_iter;
  return MSG_OK;
}

}  // namespace msg
