// msg_api.cu -- C ABI of libmsg123gpu.so: context lifecycle, state transfer, and the
// host-side control of the Newton iteration (calc_numsol) and of the time loop.
//
// The control flow restates Nonlinear_solution.f90 and Time_module.f90; every
// vector operation runs on the device and only scalars (norms, dot products, the
// arg-max of the update) cross PCIe.
#include "msg_ctx.cuh"
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <vector>
#include <deque>
#include <atomic>
#include <new>
#include <string>
#include <thread>
#include <vector>

namespace msg {

static thread_local char g_err[512] = "";
long long g_launches = 0;

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char *get_error() { return g_err; }

static constexpr double VARMAX = 1.0e3, XMAX = 1.0e4, DSMAL = 1.0e-20;
static constexpr double MACHI_EPS = 1.1920928955078125e-07;   // epsilon(1._SP)

static int nblk(int n) { return (n + kThreads - 1) / kThreads; }

__global__ void k_fill(int n, double *y, double v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = v;
}
__global__ void k_scale_copy(int n, double *y, const double *x, double a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = __dmul_rn(x[i], a);
}
// outjvec = -(f2 - f1) * eps_inv  (calc_vecjacf, Calc_function.f90:613-617)
// Newton initial guess: h = h_old + ratio*(h_old - h_old2)
__global__ void k_extrap(int n, double *h, const double *h_old, const double *h_old2, double ratio) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    h[i] = __dadd_rn(h_old[i], __dmul_rn(ratio, __dsub_rn(h_old[i], h_old2[i])));
}
// out = -(f2 - f1) / eps; with NEG the caller passes g = -f1, and f2 - f1 = f2 + g exactly.
template <bool NEG>
__global__ void k_vecjac_out(int n, double *out, const double *f2, const double *f1, double eps_inv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = __dmul_rn(-(NEG ? __dadd_rn(f2[i], f1[i]) : __dsub_rn(f2[i], f1[i])), eps_inv);
}
__global__ void k_to_f32(size_t n, const double *a, float *b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void k_csr_to_dia(int nx, int ny, int nz, const int *offind, const double *lumat, double *lu) {
  int N = nx * ny * nz, nxy = nx * ny;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int iz = i / nxy, rem = i - iz * nxy, iy = rem / nx, ix = rem - iy * nx;
  const bool has[6] = {iz > 0, iy > 0, ix > 0, ix < nx - 1, iy < ny - 1, iz < nz - 1};
  int k = offind[i];
  for (int d = 0; d < 6; ++d) lu[(size_t)d * N + i] = has[d] ? lumat[k++] : 0.0;
}

static double sum_part(msg_ctx *c, int count, int *rc) {
  double v = 0.0;
  *rc = finish(c, count, 1, &v);
  return v;
}

// calc_func + its squared norm
static int func_norm(msg_ctx *c, const double *h, double *F, double *l2) {
  if (c->timing) cudaEventRecord(c->ev[7], c->stream);
  int rc = launch_calc_func(c, h, F, true);
  if (rc) return rc;
  *l2 = sum_part(c, flux_parts(c), &rc);   // synchronises the stream
  c->l2_last = *l2;
  if (c->timing) {
    cudaEventRecord(c->ev[0], c->stream);
    cudaEventSynchronize(c->ev[0]);
    float a = 0.f;
    cudaEventElapsedTime(&a, c->ev[7], c->ev[0]);
    c->t_ms[3] += a;
  }
  return rc;
}

// make_matvec (Make_linearsystem.f90:24-68) + AMG setup when requested.  reuse: the last
// residual evaluation was at head_new (true from the second Newton iteration on).
// assembled: the line search already assembled the system at head_new (asm_ahead), so only
// the hierarchy decision remains.
static int make_matvec(msg_ctx *c, double *l2_rhs, bool reuse, bool assembled = false) {
  cudaEvent_t *ev = c->ev;
  if (c->timing) cudaEventRecord(ev[0], c->stream);
  int rc = assembled ? MSG_OK : launch_make_matvec(c, reuse);
  if (rc) return rc;
  if (l2_rhs) {   // ||F||^2 (a host round trip; calc_numsol needs it at its first iteration only)
    *l2_rhs = sum_part(c, flux_parts(c), &rc);
    if (rc) return rc;
  }
  if (c->timing) cudaEventRecord(ev[1], c->stream);
  if (c->prm.precon_type == 1 && !c->prm.ref_quirks) {
    // amg_lag = k >= 1: the hierarchy built at a time step's first Newton iteration is
    // kept for that step and the next k-1 steps (the level-1 smoother always uses the
    // current Jacobian)
    if (!c->prm.amg_lag || c->amg_nlevel <= 1 || c->amg_force || (c->out_iter <= 1 && c->amg_age >= c->prm.amg_lag)) {
      if ((rc = amg_setup(c))) return rc;
      c->amg_age = 0;
      c->amg_force = 0;
    }
  }
  if (c->timing) {
    cudaEventRecord(ev[2], c->stream);
    cudaEventSynchronize(ev[2]);
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, ev[0], ev[1]);
    cudaEventElapsedTime(&b, ev[1], ev[2]);
    c->t_ms[0] += a; c->t_ms[2] += b;
  }
  return MSG_OK;
}

static int solve_linalg(msg_ctx *c, double init_norm, double *x, double *last_norm, bool x_zero = false) {
  if (c->timing) cudaEventRecord(c->ev[3], c->stream);
  c->bnorm = init_norm;
  int rc = solve_bicgs(c, x, x_zero);
  if (rc) return rc;
  *last_norm = c->rnorm;
  if (c->timing) {
    cudaEventRecord(c->ev[4], c->stream);
    cudaEventSynchronize(c->ev[4]);
    float a = 0.f;
    cudaEventElapsedTime(&a, c->ev[3], c->ev[4]);
    c->t_ms[1] += a;
  }
  return MSG_OK;
}

// calc_vecjacf (Calc_function.f90:515-621).  neg_f1, when given, is -F(x) already at hand:
// the make_matvec right-hand side of the iterate x it was assembled at, whose arithmetic is
// that of calc_func term for term, so the finite difference is the same bit for bit and
// one residual evaluation is saved.
static int vecjacf(msg_ctx *c, const double *x, const double *v, double *out, const double *neg_f1 = nullptr) {
  const int n = c->N;
  const double *f1 = neg_f1;
  double *f2 = c->t, *jc = c->z;
  int rc;
  double dummy;
  if (!f1) {
    if ((rc = func_norm(c, x, c->v, &dummy))) return rc;
    f1 = c->v;
  }
  double l2_v, l2_x, l1_v;
  if ((rc = dot(c, v, v, n, &l2_v))) return rc;
  if ((rc = dot(c, x, v, n, &l2_x))) return rc;
  if ((rc = norm1(c, v, n, &l1_v))) return rc;
  double sign = (l2_x < 0.0) ? -1.0 : 1.0;
  double eps = sign * std::sqrt(MACHI_EPS) * std::fmax(std::fabs(l2_x), l1_v) / l2_v;
  double eps_inv = 1.0 / eps;
  if ((rc = axpby(c, jc, x, eps, v, n))) return rc;
  if ((rc = func_norm(c, jc, f2, &dummy))) return rc;
  if (neg_f1) k_vecjac_out<true><<<nblk(n), 256, 0, c->stream>>>(n, out, f2, f1, eps_inv);
  else k_vecjac_out<false><<<nblk(n), 256, 0, c->stream>>>(n, out, f2, f1, eps_inv);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

static int calc_funcl2norm(msg_ctx *c, double in_lam) {
  c->asm_ahead = 0;   // head_new moves off the point the system was assembled at
  c->head_moved = 1;
  int rc = axpby(c, c->head_new, c->head_pre, in_lam, c->head_change, c->N);
  if (rc) return rc;
  return func_norm(c, c->head_new, c->new_f, &c->l2_new);
}

// run_backtr (Nonlinear_solution.f90:441-631)
// The line-search slope reads the right-hand side assembled for this Newton iteration,
// which nothing changes before the slope is taken -- except with the reference's AMG
// quirks, where the preconditioner leaves its input there (Q2) and slope_rhs holds it.
static bool slope_from_rhs(const msg_ctx *c) { return !(c->prm.precon_type == 1 && c->prm.ref_quirks); }

static int run_backtr(msg_ctx *c) {
  const int n = c->N;
  const double back_alpha = 1.0e-4, back_beta = 0.9;
  double l2_new2 = c->l2_new, lam2 = 1.0, maxpnorm = 1.0, lam_len = 1.0;
  double temp_lam, rhs1, rhs2, lam_inv, lam2_inv, del_lam, av, bv, root, lam_max, lam_base, lam_diff, lam_incr;
  int rc;
  c->lam = 1.0;
  // J.dh by finite differences at the iterate the system was assembled at (rhs = -F there),
  // taken before F(head_new) so that the last residual evaluation of the line search is
  // always the one at the accepted head_new (its S and kr stay current; calc_numsol reuses it)
  double *jacvec = c->tmpv;
  // J.dh of the assembled Jacobian (jv_mode 1): BiCGStab started from dh = 0 and keeps
  // r = rhs - J dh, so the slope below is (rhs, rhs - r), formed in one pass
  const bool jv_resid = c->prm.jv_mode == 1 && !c->prm.ref_quirks;
  if (!jv_resid && (rc = vecjacf(c, c->head_pre, c->head_change, jacvec, c->rhs))) return rc;
  // F(head_new) and its norm in the flux pass's order (l2_last, what calc_numsol keeps), the
  // norm collected with the statistics below in one host round trip (timed runs take it
  // through func_norm, which records the residual's time)
  //
  // Assembly ahead: unless the line search backtracks, the next Newton iteration assembles
  // the system at this same head_new, and the assembly pass computes F(head_new) (as -F in
  // its right-hand side, term for term the residual pass's arithmetic, with the same F^2
  // partials) and S, kr and the storage term there.  So the residual evaluation at the
  // full step is the assembly itself, into rhs_alt (the current rhs is still needed for the
  // slope): one van Genuchten and one flux pass per Newton iteration fewer.  Not with the
  // convergence log (it records this iteration's dmat), the phase timers or the reference's
  // quirks.
  const bool ahead = !c->timing && !c->clog_on && !c->prm.ref_quirks;
  const double *fnew = c->new_f;
  if (c->timing) {
    double dummy;
    if ((rc = func_norm(c, c->head_new, c->new_f, &dummy))) return rc;
  } else if (ahead) {
    if ((rc = launch_make_matvec(c, false, c->rhs_alt))) return rc;
    if ((rc = finish_to(c, flux_parts(c), 1, 4))) return rc;
    fnew = c->rhs_alt;   // -F: the same squares
    c->asm_ahead = 1;
  } else {
    if ((rc = launch_calc_func(c, c->head_new, c->new_f, true))) return rc;
    if ((rc = finish_to(c, flux_parts(c), 1, 4))) return rc;
  }
  // ||dh||^2, ||F(head_new)||^2, the slope and lam_length in one pass; lam_length is taken
  // again if dh is shortened (the slope, from J dh of the unshortened step, is scaled below)
  const double *srhs = slope_from_rhs(c) ? c->rhs : c->slope_rhs;   // or (Q2) the last preconditioner input
  double stats[5];
  if ((rc = backtr_stats(c, c->head_change, c->head_new, fnew, srhs, jv_resid ? nullptr : jacvec, c->rhs, c->r,
                         stats, !c->timing)))
    return rc;
  if (!c->timing) c->l2_last = stats[4];
  const double l2_pnorm = stats[0];
  c->l2_new = stats[1];
  double slope = stats[2];
  lam_len = stats[3];
  double sql2_pnorm = std::sqrt(l2_pnorm);
  bool scaled = false;
  if (sql2_pnorm > c->maxstep) {
    maxpnorm = c->maxstep / sql2_pnorm;
    if ((rc = scale(c, c->head_change, maxpnorm, n))) return rc;
    sql2_pnorm = c->maxstep;
    scaled = true;
  }
  double step_len = sql2_pnorm;
  slope = slope * maxpnorm;
  if (scaled && (rc = lam_length(c, c->head_change, c->head_new, &lam_len))) return rc;
  c->l2_jnorm = c->l2_jnorm * maxpnorm * maxpnorm;
  double step_tol = std::pow(MACHI_EPS, 2.0 / 3.0);
  double lam_min = step_tol / lam_len;
  double alpha_cond = 0.5 * c->l2_pre + back_alpha * c->lam * slope, beta_cond;
  c->gradient = slope;
  for (;;) {
    if (0.5 * c->l2_new <= alpha_cond) break;
    c->back_iter++;
    if ((rc = calc_funcl2norm(c, c->lam))) return rc;
    if (c->lam == 1.0) {
      temp_lam = -slope / (2.0 * (0.5 * c->l2_new - 0.5 * c->l2_pre - slope));
    } else {
      rhs1 = 0.5 * c->l2_new - 0.5 * c->l2_pre - c->lam * slope;
      rhs2 = l2_new2 - 0.5 * c->l2_pre - lam2 * slope;
      lam_inv = 1.0 / (c->lam * c->lam);
      lam2_inv = 1.0 / (lam2 * lam2);
      del_lam = 1.0 / (c->lam - lam2);
      av = (rhs1 * lam_inv - rhs2 * lam2_inv) * del_lam;
      bv = (-lam2 * rhs1 * lam_inv + c->lam * rhs2 * lam2_inv) * del_lam;
      if (av == 0) {
        temp_lam = -slope / (2.0 * bv);
      } else {
        root = bv * bv - 3.0 * av * slope;
        if (root < 0.0) temp_lam = 0.5 * c->lam;
        else if (bv <= 0.0) temp_lam = (-bv + std::sqrt(root)) / (3.0 * av);
        else temp_lam = -slope / (bv + std::sqrt(root));
        if (temp_lam > 0.5 * c->lam) temp_lam = 0.5 * c->lam;
      }
    }
    lam2 = c->lam;
    l2_new2 = 0.5 * c->l2_new;
    c->lam = std::fmax(temp_lam, 0.1 * c->lam);
    if (c->lam < lam_min) { c->back_flag = 1; return MSG_OK; }
    alpha_cond = 0.5 * c->l2_pre + back_alpha * c->lam * slope;
  }
  alpha_cond = 0.5 * c->l2_pre + back_alpha * c->lam * slope;
  beta_cond = 0.5 * c->l2_pre + back_beta * c->lam * slope;
  if (0.5 * c->l2_new < beta_cond) {
    if (c->lam == 1.0 && sql2_pnorm < step_len) {
      lam_max = step_len / sql2_pnorm;
      for (;;) {
        if (0.5 * c->l2_new > alpha_cond || 0.5 * c->l2_new >= beta_cond || c->lam >= lam_max) break;
        lam2 = c->lam; l2_new2 = 0.5 * c->l2_new; c->lam = std::fmin(2.0 * c->lam, lam_max);
        if ((rc = calc_funcl2norm(c, c->lam))) return rc;
        alpha_cond = 0.5 * c->l2_pre + back_alpha * c->lam * slope;
        beta_cond = 0.5 * c->l2_pre + back_beta * c->lam * slope;
      }
    }
    if (c->lam < 1.0 || (c->lam > 1.0 && 0.5 * c->l2_new > alpha_cond)) {
      lam_base = std::fmin(c->lam, lam2);
      lam_diff = std::fabs(lam2 - c->lam);
      for (;;) {
        if (0.5 * c->l2_new <= alpha_cond && (0.5 * c->l2_new >= beta_cond || lam_diff <= lam_min)) break;
        lam_incr = 0.5 * lam_diff;
        c->lam = lam_base + lam_incr;
        if ((rc = calc_funcl2norm(c, c->lam))) return rc;
        alpha_cond = 0.5 * c->l2_pre + back_alpha * c->lam * slope;
        beta_cond = 0.5 * c->l2_pre + back_beta * c->lam * slope;
        if (0.5 * c->l2_new > alpha_cond) lam_diff = lam_incr;
        else if (0.5 * c->l2_new < beta_cond) { lam_base = c->lam; lam_diff = lam_diff - lam_incr; }
        if (lam_diff == 0.0) break;
      }
      if (0.5 * c->l2_new < beta_cond) {
        if ((rc = calc_funcl2norm(c, lam_base))) return rc;
        c->beta_iter++;
      }
      if (c->beta_iter == 10) { c->back_flag = 1; return MSG_OK; }
    }
  }
  (void)l2_new2;
  return MSG_OK;
}

// set_eater (Nonlinear_solution.f90:414-439)
static void set_eater(msg_ctx *c) {
  const double eta_max = 0.9, eta_min = 1.0e-4, eta_alpha = (1.0 + std::sqrt(5.0)) / 2.0;
  double eta_safe = std::pow(c->eta, eta_alpha);
  double minus1 = 1.0 - c->lam;
  double lin = std::sqrt(minus1 * minus1 * c->l2_pre + 2.0 * c->lam * minus1 * c->gradient + c->lam * c->lam * c->l2_jnorm);
  c->eta = std::fabs(std::sqrt(c->l2_new) - lin) / std::sqrt(c->l2_pre);
  if (eta_safe < 0.1) eta_safe = 0.0;
  c->eta = std::fmax(c->eta, eta_safe);
  c->eta = std::fmax(c->eta, eta_min);
  c->eta = std::fmin(c->eta, eta_max);
}

static int copy_d2d(msg_ctx *c, double *dst, const double *src, int n) {
  MSG_CUDA(cudaMemcpyAsync(dst, src, (size_t)n * 8, cudaMemcpyDeviceToDevice, c->stream));
  return MSG_OK;
}

constexpr size_t kConvLogMax = (size_t)1 << 20;
using ConvLog = std::deque<msg_convrec_t>;

// One line of the convergence log (Nonlinear_solution.f90:240-252): the values at the
// cell of the largest change, scaled as the reference writes them.
static int convlog_push(msg_ctx *c, int maxnun) {
  msg_convrec_t r;
  memset(&r, 0, sizeof(r));
  r.time = c->current_t; r.delt = c->delt;
  r.out_iter = c->out_iter; r.in_iter = c->in_iter; r.back_iter = c->back_iter;
  r.cell = maxnun;
  r.maxvar = c->maxvar * c->len_scal;
  r.status = -1;
  if (maxnun >= 1 && maxnun <= c->N) {
    double v[3];
    MSG_CUDA(cudaMemcpyAsync(&v[0], c->dmat + (maxnun - 1), 8, cudaMemcpyDeviceToHost, c->stream));
    MSG_CUDA(cudaMemcpyAsync(&v[1], c->rhs + (maxnun - 1), 8, cudaMemcpyDeviceToHost, c->stream));
    MSG_CUDA(cudaMemcpyAsync(&v[2], c->head_new + (maxnun - 1), 8, cudaMemcpyDeviceToHost, c->stream));
    MSG_CUDA(cudaStreamSynchronize(c->stream));
    // len_scal is real(SP) in the reference, so len_scal**2 and **3 are single-precision
    // products (Nonlinear_solution.f90:245-247) before they scale the double values
    const float Lf = (float)c->len_scal;
    const float L2 = Lf * Lf, L3 = L2 * Lf;
    r.dmat = v[0] * (double)L2;
    r.rhs = v[1] * (double)L3;
    r.head = v[2] * c->len_scal;
  }
  ConvLog &q = *reinterpret_cast<ConvLog *>(c->clog);
  if (q.size() >= kConvLogMax) q.pop_front();
  q.push_back(r);
  return MSG_OK;
}

// calc_numsol (Nonlinear_solution.f90:33-294)
static int calc_numsol(msg_ctx *c, msg_stats_t *stx) {
  const int n = c->N;
  int rc, maxnun = 0, status = MSG_NEWTON_MAXIT, nan = 0;
  double maxunk, check_val;
  msg_stats_t st;
  memset(&st, 0, sizeof(st));
  double l2x;
  c->amg_age++;
  c->asm_ahead = 0;
  if ((rc = dot(c, c->head_new, c->head_new, n, &l2x))) return rc;      // set_backtr
  c->maxstep = std::sqrt(l2x) * VARMAX;
  if (c->maxstep < 1.0) c->maxstep = 1.0;
  for (c->out_iter = 1; c->out_iter <= c->prm.maxout_iter; ++c->out_iter) {
    if (c->out_iter > 1) c->l2_pre = c->l2_new;
    c->back_flag = 0; c->back_iter = 0; c->beta_iter = 0;
    double l2r = 0.0;
    // from the second iteration on, the previous iteration ended with F evaluated at
    // head_new (line search or the closing evaluation), leaving S, kr and the storage
    // term there in srat_new / kr / sto
    // the first assembly reuses S, kr and the storage term when the guess selection left
    // them at head_new (the chosen guess was the last one evaluated)
    // the previous iteration's line search assembled the system at head_new (its rhs is in
    // rhs_alt) unless it backtracked
    const bool assembled = c->asm_ahead;
    if (assembled) {
      std::swap(c->rhs, c->rhs_alt);
      c->asm_ahead = 0;
    }
    if ((rc = make_matvec(c, c->out_iter == 1 ? &l2r : nullptr, c->out_iter > 1 || c->vg_at_head, assembled)))
      return rc;
    c->vg_at_head = 0;
    if (!slope_from_rhs(c) && (rc = copy_d2d(c, c->slope_rhs, c->rhs, n))) return rc;
    if (c->out_iter == 1) { c->l2_new = l2r; c->l2_pre = c->l2_new; c->eta = 0.5; }
    // head_pre takes the iterate by a buffer swap: nothing reads head_new again before
    // head_new = head_pre + dh overwrites all of it (in check_abserrmax's pass)
    std::swap(c->head_pre, c->head_new);
    // dh starts at zero; BiCGStab's first update writes it without reading it
    if (c->prm.maxinn_iter < 1) MSG_CUDA(cudaMemsetAsync(c->head_change, 0, (size_t)n * 8, c->stream));
    c->conv_flag = 0;
    c->errtol = c->prm.lin_tol > 0 ? c->prm.lin_tol : c->eta;
    if ((rc = solve_linalg(c, c->l2_pre, c->head_change, &c->l2_jnorm, true))) return rc;   // from dh = 0
    st.inner_total += c->in_iter; st.in_iter_last = c->in_iter;
    // head_new = head_pre + dh, formed inside check_abserrmax's pass
    if ((rc = abserrmax(c, c->head_new, c->head_pre, &c->maxvar, &maxunk, &maxnun, &nan, c->head_change))) return rc;
    const double maxvar_full = c->maxvar, maxunk_full = maxunk;   // of the full step, for the line search below
    const int maxnun_full = maxnun, nan_full = nan;
    check_val = std::fabs(c->maxvar) * c->len_scal;
    maxunk = std::fabs(maxunk) * c->len_scal;
    double crit = c->prm.criteria_rel ? c->prm.criteria * maxunk : c->prm.criteria;
    if (c->conv_flag != 0 && maxunk == maxunk) {
      c->conv_flag = 0;
      if (check_val <= crit && maxunk < XMAX) c->conv_flag = 1;
    } else if (maxunk != maxunk) {
      status = MSG_NAN;
      break;
    }
    bool evaluated = false;   // F(head_new) and its norm already computed by the line search
    if (c->conv_flag != 1) {
      c->head_moved = 0;
      if ((rc = run_backtr(c))) return rc;
      evaluated = true;
      // check_abserrmax again: the same values as above unless the line search moved head_new
      if (c->head_moved) {
        if ((rc = abserrmax(c, c->head_new, c->head_pre, &c->maxvar, &maxunk, &maxnun, &nan))) return rc;
      } else {
        c->maxvar = maxvar_full; maxunk = maxunk_full; maxnun = maxnun_full; nan = nan_full;
      }
      check_val = std::fabs(c->maxvar) * c->len_scal;
      maxunk = std::fabs(maxunk) * c->len_scal;
      crit = c->prm.criteria_rel ? c->prm.criteria * maxunk : c->prm.criteria;
      if (check_val >= VARMAX || maxunk >= XMAX) c->back_flag = 1;
      else if (check_val <= crit && maxunk < XMAX) c->conv_flag = 1;
      if (c->conv_flag != 1 && c->back_flag != 1) set_eater(c);
    }
    if (evaluated) c->l2_new = c->l2_last;
    else if ((rc = func_norm(c, c->head_new, c->new_f, &c->l2_new))) return rc;
    st.back_total += c->back_iter; st.back_iter_last = c->back_iter;
    double conv_var = c->maxvar * c->len_scal;
    if (c->clog_on && (rc = convlog_push(c, maxnun))) return rc;
    if (c->conv_flag == 1) {
      if ((rc = copy_d2d(c, c->surf_head, c->head_new, c->S))) return rc;   // calc_surfw
      status = MSG_OK;
      break;
    } else if (c->back_flag == 1) {
      status = MSG_LINESEARCH_FAIL; break;
    } else if (c->out_iter == c->prm.maxout_iter) {
      status = MSG_NEWTON_MAXIT; break;
    } else if (std::fabs(conv_var) >= VARMAX || maxunk >= XMAX) {
      status = MSG_DIVERGED; break;
    }
  }
  if (c->out_iter > c->prm.maxout_iter) c->out_iter = c->prm.maxout_iter;
  if (c->clog_on && status != MSG_NAN) {   // the reference writes no line for a NaN update
    ConvLog &q = *reinterpret_cast<ConvLog *>(c->clog);
    if (!q.empty()) q.back().status = status;
  }
  st.status = status; st.out_iter = c->out_iter; st.maxnun = maxnun;
  st.maxvar = c->maxvar * c->len_scal; st.l2_new = c->l2_new;
  if (stx) *stx = st;
  return status;
}

// apply_heuri (Time_module.f90:1522-1543)
static void apply_heuri(msg_ctx *c, int out_num) {
  int incr = (int)(c->prm.maxout_iter * 0.4), decr = (int)(c->prm.maxout_iter * 0.8);
  if (out_num <= incr) c->delt = c->delt_old1 * 1.2;
  else if (out_num <= decr) c->delt = c->delt_old1;
  else c->delt = c->delt_old1 * 0.8;
}

// update_tstep / calc_nextst loop (Time_module.f90:34-273); current_t is real(SP).
static int advance(msg_ctx *c, int nsteps, double rech_until, double rech_after, msg_run_stats_t *rs) {
  msg_run_stats_t R;
  memset(&R, 0, sizeof(R));
  int conv = c->last_conv, last_out = c->last_out, status = MSG_OK, rc;
  const int n = c->N, S = c->S;
  while (R.accepted < nsteps) {
    if (conv == 1) {
      if (c->timestep_num == 0) c->delt_old1 = c->delt;
      c->timestep_num++;
      c->delt_old2 = c->delt_old1; c->delt_old1 = c->delt;
      if (c->prm.sim_type == 0) c->delt = c->delt * c->prm.inc_fact;
      else { apply_heuri(c, last_out); if (c->delt > c->prm.max_step) c->delt = c->prm.max_step; }
      if ((rc = copy_d2d(c, c->head_old2, c->head_old, n))) return rc;
      if ((rc = copy_d2d(c, c->head_old, c->head_new, n))) return rc;
      if ((rc = copy_d2d(c, c->srat_old, c->srat_new, n))) return rc;
      if ((rc = copy_d2d(c, c->surf_old, c->surf_head, S))) return rc;
    } else if (conv == 0) {
      c->current_t = (double)(float)(c->current_t - (double)(float)c->delt);
      c->delt = c->delt * 0.5;
      if ((rc = copy_d2d(c, c->head_new, c->head_old, n))) return rc;
      if ((rc = copy_d2d(c, c->srat_new, c->srat_old, n))) return rc;
      if ((rc = copy_d2d(c, c->surf_head, c->surf_old, S))) return rc;
      R.rejected++;
    }
    if (c->current_t < rech_until && c->current_t + c->delt > rech_until) c->delt = rech_until - c->current_t;
    if (c->current_t + c->delt > c->prm.end_time) c->delt = c->prm.end_time - c->current_t;
    if (c->delt < DSMAL) { status = MSG_DT_TOO_SMALL; break; }
    double sc = (c->current_t < rech_until) ? 1.0 : rech_after;
    k_scale_copy<<<nblk(S), kThreads, 0, c->stream>>>(S, c->calc_rech, c->rech_base, sc);
    MSG_CHECK_LAUNCH();
    c->current_t = (double)(float)(c->current_t + (double)(float)c->delt);
    c->delt_inv = 1.0 / c->delt;
    // update_tstep (Time_module.f90:83-87): well rates after an accepted step or at the start
    if ((conv == 1 || c->timestep_num == 0) && c->nwell > 0) {
      if ((rc = launch_wells(c))) return rc;
    }
    msg_stats_t st;
    bool learned_try = false;
    c->vg_at_head = 0;
    const bool paused = c->prm.guess_select == 2 && c->guess_skip > 0;
    if (paused) c->guess_skip--;
    if (c->prm.guess_mode == 2 && c->timestep_num > 0 && conv != 0 && learned_ready(c) && !paused) {
      if ((rc = learned_guess(c))) return rc;       // head_new <- h_old + CNN increment
      learned_try = true;
      if (c->prm.guess_select) {
        // keep the learned guess only if its residual is below the extrapolation's
        double fl = 0.0, fe = 0.0;
        if ((rc = func_norm(c, c->head_new, c->new_f, &fl))) return rc;
        k_extrap<<<nblk(n), 256, 0, c->stream>>>(n, c->head_pre, c->head_old, c->head_old2, c->delt / c->delt_old1);
        MSG_CHECK_LAUNCH();
        if ((rc = func_norm(c, c->head_pre, c->new_f, &fe))) return rc;
        if (!(fl < fe)) {
          // the extrapolation was evaluated last: its S, kr and storage serve the first assembly
          if ((rc = copy_d2d(c, c->head_new, c->head_pre, n))) return rc;
          learned_try = false;
          c->guess_rejected++;
          c->vg_at_head = 1;
          if (c->prm.guess_select == 2) {   // back off: 1, 2, 4, 8 steps without the network
            c->guess_backoff = std::min(std::max(2 * c->guess_backoff, 1), 8);
            c->guess_skip = c->guess_backoff;
          }
        } else {
          c->guess_backoff = 0;
        }
      }
    } else if (c->prm.guess_mode >= 1 && c->timestep_num > 0) {
      k_extrap<<<nblk(n), 256, 0, c->stream>>>(n, c->head_new, c->head_old, c->head_old2, c->delt / c->delt_old1);
      MSG_CHECK_LAUNCH();
    }
    rc = calc_numsol(c, &st);
    if (rc < 0) return rc;
    // A vetted learned guess (its residual beat the extrapolation's) that then fails to
    // converge points at the time step, not at the guess: the step is rejected as usual.
    // An unvetted guess, or a breakdown (NaN, divergence), is retried from the extrapolation.
    const bool breakdown = (rc == MSG_NAN || rc == MSG_DIVERGED);
    if (learned_try && rc != MSG_OK && (!c->prm.guess_select || breakdown)) {
      // fallback: the same time step again from the plain extrapolation
      R.newton_total += st.out_iter; R.krylov_total += st.inner_total; R.back_total += st.back_total;
      c->guess_fallbacks++;
      if ((rc = copy_d2d(c, c->srat_new, c->srat_old, n))) return rc;
      if ((rc = copy_d2d(c, c->surf_head, c->surf_old, S))) return rc;
      k_extrap<<<nblk(n), 256, 0, c->stream>>>(n, c->head_new, c->head_old, c->head_old2, c->delt / c->delt_old1);
      MSG_CHECK_LAUNCH();
      rc = calc_numsol(c, &st);
      if (rc < 0) return rc;
    }
    R.newton_total += st.out_iter; R.krylov_total += st.inner_total; R.back_total += st.back_total;
    last_out = st.out_iter;
    conv = (rc == MSG_OK) ? 1 : 0;
    c->last_out = last_out;
    if (conv) { R.accepted++; if (c->current_t >= c->prm.end_time) break; }
  }
  c->last_conv = conv;
  R.status = status; R.current_t = c->current_t; R.delt = c->delt;
  if (rs) *rs = R;
  return status;
}

static void free_ctx(msg_ctx *c);

}  // namespace msg

using namespace msg;

// =====================================================================================
// C ABI
// =====================================================================================
extern "C" {

const char *msg_gpu_last_error(void) { return get_error(); }

#define ALLOC(ptr, bytes) MSG_CUDA(cudaMalloc((void **)&(ptr), (bytes)))
#define UPLOAD(dst, src, bytes) MSG_CUDA(cudaMemcpyAsync((dst), (src), (bytes), cudaMemcpyHostToDevice, c->stream))

static int create_impl(msg_ctx *c, const msg_grid_t *g, const msg_params_t *p) {
  const size_t N = (size_t)g->nx * g->ny * g->nz, S = (size_t)g->nx * g->ny;
  c->nx = g->nx; c->ny = g->ny; c->nz = g->nz; c->N = (int)N; c->S = (int)S; c->nxy = (int)S;
  c->sea_top = g->sea_top; c->free_drainage = g->free_drainage;
  c->prm = *p;
  c->len_scal = p->len_scal;
  c->newper = MACHI_EPS * (double)(1.0f / (float)p->len_scal);   // Prep_calculation.f90:79
  c->newper_inv = 1.0 / c->newper;
  c->delt = p->ini_step; c->delt_inv = 1.0 / p->ini_step;
  c->last_conv = -1;
  c->blk_cell = kThreads;
  c->blk_smooth = kThreads;
  MSG_CUDA(cudaGetDevice(&c->device));
  {
    // keep freed stream-ordered allocations in the pool (the AMG hierarchy is rebuilt
    // every Newton iteration; returning memory to the OS at each sync costs ~ms)
    cudaMemPool_t pool;
    MSG_CUDA(cudaDeviceGetDefaultMemPool(&pool, c->device));
    uint64_t thr = UINT64_MAX;
    MSG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  }
  MSG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  for (int k = 0; k < 8; ++k) MSG_CUDA(cudaEventCreate(&c->ev[k]));
  // symmetric face areas are required by the face-shared DIA storage
  for (int iz = 0; iz < g->nz; ++iz)
    for (int iy = 0; iy < g->ny; ++iy)
      for (int ix = 0; ix < g->nx; ++ix) {
        size_t i = ix + (size_t)g->nx * (iy + (size_t)g->ny * iz);
        if (ix > 0 && g->face_area[2 * N + i] != g->face_area[3 * N + i - 1]) {
          set_error("face areas are not symmetric at cell %zu (west/east)", i);
          return MSG_ERR_ARG;
        }
        if (iy > 0 && g->face_area[1 * N + i] != g->face_area[4 * N + i - g->nx]) {
          set_error("face areas are not symmetric at cell %zu (north/south)", i);
          return MSG_ERR_ARG;
        }
        if (iz > 0 && g->face_area[0 * N + i] != g->face_area[5 * N + i - S]) {
          set_error("face areas are not symmetric at cell %zu (up/down)", i);
          return MSG_ERR_ARG;
        }
      }
  float **fp[] = {&c->reta, &c->retn, &c->resi, &c->poro, &c->ss, &c->ksz};
  const float *fs[] = {g->reta, g->retn, g->resi, g->poro, g->ss, g->ksz};
  for (int k = 0; k < 6; ++k) { ALLOC(*fp[k], N * 4); UPLOAD(*fp[k], fs[k], N * 4); }
  ALLOC(c->cell_top, N * 8); UPLOAD(c->cell_top, g->cell_top, N * 8);
  ALLOC(c->cell_vol, N * 8); UPLOAD(c->cell_vol, g->cell_vol, N * 8);
  ALLOC(c->hy, 3 * N * 8); ALLOC(c->ab, 3 * N * 8); ALLOC(c->invd, 3 * N * 8);
  double **sp[] = {&c->surf_top, &c->surf_bott, &c->surf_reli, &c->surf_parm, &c->read_seal};
  const double *ss_[] = {g->surf_top, g->surf_bott, g->surf_reli, g->surf_parm, g->sea_head};
  for (int k = 0; k < 5; ++k) {
    ALLOC(*sp[k], S * 8);
    if (ss_[k]) UPLOAD(*sp[k], ss_[k], S * 8);
    else MSG_CUDA(cudaMemsetAsync(*sp[k], 0, S * 8, c->stream));
  }
  double **sz[] = {&c->hydf_surf, &c->abyd_surf, &c->calc_rech, &c->rech_base, &c->sea_hydf, &c->sea_abyd,
                   &c->drain, &c->surf_head, &c->surf_old, &c->top_invd};
  for (auto q : sz) { ALLOC(*q, S * 8); MSG_CUDA(cudaMemsetAsync(*q, 0, S * 8, c->stream)); }
  ALLOC(c->offind, (N + 1) * 4);
  double **vn[] = {&c->head_new, &c->head_old, &c->head_old2, &c->head_pre, &c->head_change, &c->srat_new, &c->srat_old,
                   &c->new_f, &c->kr, &c->kr_per, &c->alp, &c->sto, &c->stod, &c->tmpv, &c->dmat, &c->rhs,
                   &c->slope_rhs, &c->rhs_alt, &c->dilu_d, &c->r, &c->rs, &c->p, &c->v, &c->t, &c->z};
  for (auto q : vn) { ALLOC(*q, N * 8); MSG_CUDA(cudaMemsetAsync(*q, 0, N * 8, c->stream)); }
  ALLOC(c->lu, 6 * N * 8);
  if (p->precision == 1) {
    ALLOC(c->dmat_f, N * 4);
    ALLOC(c->lu_f, 6 * N * 4);
  }
  // up to four arrays of one partial per block of 256 cells (the line search's k_backtr_stats)
  size_t npart = std::max((size_t)kRedBlocks * 8, 4 * (size_t)nblk((int)N) + 64);
  // the flux passes' 3D grid can have more blocks than nblk(N) when nx or ny is not a
  // multiple of the tile (32 x 8)
  npart = std::max(npart, (size_t)((g->nx + 31) / 32) * ((g->ny + 7) / 8) * g->nz + 64);
  ALLOC(c->part, npart * 8);
  c->npart = npart;
  ALLOC(c->dres, 16 * 8);
  MSG_CUDA(cudaMallocHost((void **)&c->hpin, (size_t)kRedBlocks * 8 * 8));
  int rc = build_connectivity(c, g);
  if (rc) return rc;
  if (p->precon_type == 0 || p->ref_quirks) {
    if ((rc = build_wavefront(c))) return rc;
  }
  if (p->precon_type == 1 && !p->ref_quirks) {
    if ((rc = amg_reserve(c))) return rc;
  }
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  return MSG_OK;
}

int msg_gpu_create(const msg_grid_t *grid, const msg_params_t *params, msg_ctx_t **out) {
  if (!grid || !params || !out) { set_error("null argument"); return MSG_ERR_ARG; }
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1) { set_error("empty grid"); return MSG_ERR_SIZE; }
  if ((double)grid->nx * grid->ny * grid->nz > 2.0e9 / 6.0) { set_error("grid too large for int32 CSR"); return MSG_ERR_SIZE; }
  if (params->len_scal <= 0 || params->ini_step <= 0) { set_error("len_scal and ini_step must be positive"); return MSG_ERR_ARG; }
  if (params->maxout_iter < 1 || params->maxinn_iter < 1) { set_error("iteration caps must be >= 1"); return MSG_ERR_ARG; }
  if (params->vg_form != 0 && params->vg_form != 1) { set_error("vg_form must be 0 or 1"); return MSG_ERR_ARG; }
  if (params->precision != 0 && params->precision != 1) { set_error("precision must be 0 or 1"); return MSG_ERR_ARG; }
  if (params->jv_mode != 0 && params->jv_mode != 1) { set_error("jv_mode must be 0 or 1"); return MSG_ERR_ARG; }
  if (params->guess_select < 0 || params->guess_select > 2) { set_error("guess_select must be 0, 1 or 2"); return MSG_ERR_ARG; }
  const void *req[] = {grid->reta, grid->retn, grid->resi, grid->poro, grid->ss, grid->ksx, grid->ksy, grid->ksz,
                       grid->cell_top, grid->cell_vol, grid->dis2face, grid->face_area, grid->surf_top, grid->surf_bott};
  for (auto q : req) if (!q) { set_error("required grid array is NULL"); return MSG_ERR_ARG; }
  msg_ctx *c = new (std::nothrow) msg_ctx();
  if (!c) { set_error("out of host memory"); return MSG_ERR_ARG; }
  memset(c, 0, sizeof(*c));
  int rc = create_impl(c, grid, params);
  if (rc) { free_ctx(c); return rc; }
  *out = c;
  return MSG_OK;
}

void msg_gpu_destroy(msg_ctx_t *c) {
  if (c) free_ctx(c);
}

int msg_gpu_get_connect(msg_ctx_t *c, int32_t *offind, int32_t *offrow, int32_t *conn_dir, int32_t *left_off,
                        int32_t *right_off, double *hydf_conn, double *abyd_conn, int32_t *nnz) {
  if (!c) return MSG_ERR_ARG;
  size_t M = c->nnz;
  if (offind) MSG_CUDA(cudaMemcpy(offind, c->offind, (c->N + 1) * 4, cudaMemcpyDeviceToHost));
  if (offrow) MSG_CUDA(cudaMemcpy(offrow, c->offrow, M * 4, cudaMemcpyDeviceToHost));
  if (conn_dir) MSG_CUDA(cudaMemcpy(conn_dir, c->conn_dir, M * 4, cudaMemcpyDeviceToHost));
  if (left_off) MSG_CUDA(cudaMemcpy(left_off, c->left_off, M * 4, cudaMemcpyDeviceToHost));
  if (right_off) MSG_CUDA(cudaMemcpy(right_off, c->right_off, M * 4, cudaMemcpyDeviceToHost));
  if (hydf_conn) MSG_CUDA(cudaMemcpy(hydf_conn, c->hydf_conn, M * 8, cudaMemcpyDeviceToHost));
  if (abyd_conn) MSG_CUDA(cudaMemcpy(abyd_conn, c->abyd_conn, M * 8, cudaMemcpyDeviceToHost));
  if (nnz) *nnz = c->nnz;
  return MSG_OK;
}

int msg_gpu_init_state(msg_ctx_t *c, const double *head, double delt) {
  if (!c || !head || delt <= 0) return MSG_ERR_ARG;
  size_t N = c->N, S = c->S;
  UPLOAD(c->head_new, head, N * 8);
  MSG_CUDA(cudaMemcpyAsync(c->head_old, c->head_new, N * 8, cudaMemcpyDeviceToDevice, c->stream));
  MSG_CUDA(cudaMemcpyAsync(c->head_old2, c->head_new, N * 8, cudaMemcpyDeviceToDevice, c->stream));
  int rc = launch_srat_rperm(c, c->head_new, 0.0, c->srat_old, c->kr, nullptr);
  if (rc) return rc;
  MSG_CUDA(cudaMemcpyAsync(c->srat_new, c->srat_old, N * 8, cudaMemcpyDeviceToDevice, c->stream));
  MSG_CUDA(cudaMemcpyAsync(c->surf_head, c->head_new, S * 8, cudaMemcpyDeviceToDevice, c->stream));
  MSG_CUDA(cudaMemcpyAsync(c->surf_old, c->head_new, S * 8, cudaMemcpyDeviceToDevice, c->stream));
  c->delt = delt; c->delt_inv = 1.0 / delt;
  c->current_t = 0.0; c->timestep_num = 0; c->delt_old1 = 0.0; c->last_conv = -1; c->last_out = 0;
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  return MSG_OK;
}

int msg_gpu_set_state(msg_ctx_t *c, const double *head_new, const double *head_old, const double *srat_old,
                      const double *surf_head, double delt) {
  if (!c) return MSG_ERR_ARG;
  size_t N = c->N, S = c->S;
  if (head_new) UPLOAD(c->head_new, head_new, N * 8);
  if (head_old) UPLOAD(c->head_old, head_old, N * 8);
  if (srat_old) UPLOAD(c->srat_old, srat_old, N * 8);
  if (surf_head) { UPLOAD(c->surf_head, surf_head, S * 8); UPLOAD(c->surf_old, surf_head, S * 8); }
  if (delt > 0) { c->delt = delt; c->delt_inv = 1.0 / delt; }
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  return MSG_OK;
}

int msg_gpu_copy_state(msg_ctx_t *dst, const msg_ctx_t *src) {
  if (!dst || !src) { set_error("copy_state: null context"); return MSG_ERR_ARG; }
  if (dst->nx != src->nx || dst->ny != src->ny || dst->nz != src->nz) {
    set_error("copy_state: grids differ (%dx%dx%d vs %dx%dx%d)", dst->nx, dst->ny, dst->nz, src->nx, src->ny, src->nz);
    return MSG_ERR_SIZE;
  }
  if (dst->device != src->device) { set_error("copy_state: contexts on different devices"); return MSG_ERR_ARG; }
  const size_t N = dst->N, S = dst->S;
  MSG_CUDA(cudaStreamSynchronize(src->stream));
  struct { double *d; const double *s; size_t n; } cp[] = {
      {dst->head_new, src->head_new, N}, {dst->head_old, src->head_old, N}, {dst->head_old2, src->head_old2, N},
      {dst->srat_new, src->srat_new, N}, {dst->srat_old, src->srat_old, N}, {dst->surf_head, src->surf_head, S},
      {dst->surf_old, src->surf_old, S}, {dst->calc_rech, src->calc_rech, S}, {dst->rech_base, src->rech_base, S}};
  for (auto &q : cp)
    MSG_CUDA(cudaMemcpyAsync(q.d, q.s, q.n * 8, cudaMemcpyDeviceToDevice, dst->stream));
  dst->current_t = src->current_t;
  dst->delt = src->delt; dst->delt_inv = src->delt_inv;
  dst->delt_old1 = src->delt_old1; dst->delt_old2 = src->delt_old2;
  dst->timestep_num = src->timestep_num; dst->last_conv = src->last_conv; dst->last_out = src->last_out;
  // dst's own well table applied to the copied head (as at the start of the step)
  if (dst->nwell > 0) {
    int rc = launch_wells(dst);
    if (rc) return rc;
  }
  MSG_CUDA(cudaStreamSynchronize(dst->stream));
  return MSG_OK;
}

int msg_gpu_get_state(msg_ctx_t *c, double *head_new, double *head_old, double *srat_new, double *srat_old,
                      double *surf_head) {
  if (!c) return MSG_ERR_ARG;
  size_t N = c->N, S = c->S;
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  if (head_new) MSG_CUDA(cudaMemcpy(head_new, c->head_new, N * 8, cudaMemcpyDeviceToHost));
  if (head_old) MSG_CUDA(cudaMemcpy(head_old, c->head_old, N * 8, cudaMemcpyDeviceToHost));
  if (srat_new) MSG_CUDA(cudaMemcpy(srat_new, c->srat_new, N * 8, cudaMemcpyDeviceToHost));
  if (srat_old) MSG_CUDA(cudaMemcpy(srat_old, c->srat_old, N * 8, cudaMemcpyDeviceToHost));
  if (surf_head) MSG_CUDA(cudaMemcpy(surf_head, c->surf_head, S * 8, cudaMemcpyDeviceToHost));
  return MSG_OK;
}

int msg_gpu_set_recharge(msg_ctx_t *c, const double *calc_rech) {
  if (!c || !calc_rech) return MSG_ERR_ARG;
  UPLOAD(c->rech_base, calc_rech, (size_t)c->S * 8);
  UPLOAD(c->calc_rech, calc_rech, (size_t)c->S * 8);
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  return MSG_OK;
}

int msg_gpu_srat_rperm(msg_ctx_t *c, const double *pres, double pertur, double *srat, double *rperm, double *sstor) {
  if (!c || !pres) return MSG_ERR_ARG;
  size_t N = c->N;
  UPLOAD(c->tmpv, pres, N * 8);
  int rc = launch_srat_rperm(c, c->tmpv, pertur, c->v, c->t, c->z);
  if (rc) return rc;
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  if (srat) MSG_CUDA(cudaMemcpy(srat, c->v, N * 8, cudaMemcpyDeviceToHost));
  if (rperm) MSG_CUDA(cudaMemcpy(rperm, c->t, N * 8, cudaMemcpyDeviceToHost));
  if (sstor) MSG_CUDA(cudaMemcpy(sstor, c->z, N * 8, cudaMemcpyDeviceToHost));
  return MSG_OK;
}

int msg_gpu_calc_func(msg_ctx_t *c, const double *infx, double *funcv) {
  if (!c || !infx || !funcv) return MSG_ERR_ARG;
  size_t N = c->N;
  UPLOAD(c->tmpv, infx, N * 8);
  int rc = launch_calc_func(c, c->tmpv, c->new_f, false);
  if (rc) return rc;
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  MSG_CUDA(cudaMemcpy(funcv, c->new_f, N * 8, cudaMemcpyDeviceToHost));
  return MSG_OK;
}

int msg_gpu_make_matvec(msg_ctx_t *c, double *dmat, double *lumat, double *rhs) {
  if (!c) return MSG_ERR_ARG;
  c->amg_force = 1;   // a direct call always rebuilds the hierarchy
  double l2;
  int rc = make_matvec(c, &l2, false);
  if (rc) return rc;
  size_t N = c->N;
  if (lumat) {
    double *tmp = nullptr;
    ALLOC(tmp, (size_t)c->nnz * 8);
    if ((rc = launch_dia_to_csr(c, tmp))) return rc;
    MSG_CUDA(cudaStreamSynchronize(c->stream));
    MSG_CUDA(cudaMemcpy(lumat, tmp, (size_t)c->nnz * 8, cudaMemcpyDeviceToHost));
    cudaFree(tmp);
  }
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  if (dmat) MSG_CUDA(cudaMemcpy(dmat, c->dmat, N * 8, cudaMemcpyDeviceToHost));
  if (rhs) MSG_CUDA(cudaMemcpy(rhs, c->rhs, N * 8, cudaMemcpyDeviceToHost));
  return MSG_OK;
}

int msg_gpu_set_system(msg_ctx_t *c, const double *dmat, const double *lumat, const double *rhs) {
  if (!c || !dmat || !lumat || !rhs) return MSG_ERR_ARG;
  size_t N = c->N;
  UPLOAD(c->dmat, dmat, N * 8);
  UPLOAD(c->rhs, rhs, N * 8);
  double *tmp = nullptr;
  ALLOC(tmp, (size_t)c->nnz * 8);
  UPLOAD(tmp, lumat, (size_t)c->nnz * 8);
  k_csr_to_dia<<<nblk(c->N), kThreads, 0, c->stream>>>(c->nx, c->ny, c->nz, c->offind, tmp, c->lu);
  MSG_CHECK_LAUNCH();
  if (c->dmat_f) {
    k_to_f32<<<kRedBlocks, kThreads, 0, c->stream>>>(N, c->dmat, c->dmat_f);
    MSG_CHECK_LAUNCH();
    k_to_f32<<<kRedBlocks, kThreads, 0, c->stream>>>(6 * N, c->lu, c->lu_f);
    MSG_CHECK_LAUNCH();
  }
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(tmp);
  MSG_CUDA(cudaMemcpyAsync(c->slope_rhs, c->rhs, N * 8, cudaMemcpyDeviceToDevice, c->stream));
  if (c->prm.precon_type == 1 && !c->prm.ref_quirks) {
    int rc = amg_setup(c);
    if (rc) return rc;
  }
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  return MSG_OK;
}

int msg_gpu_precond(msg_ctx_t *c, const double *r, double *z) {
  if (!c || !r || !z) return MSG_ERR_ARG;
  size_t N = c->N;
  int rc;
  if (c->prm.precon_type == 0 || c->prm.ref_quirks) {
    if ((rc = launch_precon_dilu(c))) return rc;
  }
  UPLOAD(c->tmpv, r, N * 8);
  if ((rc = apply_prec(c, c->tmpv, c->z))) return rc;
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  MSG_CUDA(cudaMemcpy(z, c->z, N * 8, cudaMemcpyDeviceToHost));
  return MSG_OK;
}

int msg_gpu_solve_linalg(msg_ctx_t *c, double init_norm, double errtol, double *inx, double *last_norm,
                         int32_t *in_iter, int32_t *conv_flag) {
  if (!c || !inx) return MSG_ERR_ARG;
  size_t N = c->N;
  UPLOAD(c->head_change, inx, N * 8);
  c->errtol = errtol;
  double ln = 0.0;
  int rc = solve_linalg(c, init_norm, c->head_change, &ln);
  if (rc) return rc;
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  MSG_CUDA(cudaMemcpy(inx, c->head_change, N * 8, cudaMemcpyDeviceToHost));
  if (last_norm) *last_norm = ln;
  if (in_iter) *in_iter = c->in_iter;
  if (conv_flag) *conv_flag = c->conv_flag;
  return MSG_OK;
}

int msg_gpu_vecjacf(msg_ctx_t *c, const double *x, const double *v, double *out) {
  if (!c || !x || !v || !out) return MSG_ERR_ARG;
  size_t N = c->N;
  UPLOAD(c->head_pre, x, N * 8);
  UPLOAD(c->head_change, v, N * 8);
  int rc = vecjacf(c, c->head_pre, c->head_change, c->tmpv);
  if (rc) return rc;
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  MSG_CUDA(cudaMemcpy(out, c->tmpv, N * 8, cudaMemcpyDeviceToHost));
  return MSG_OK;
}

int msg_gpu_calc_numsol(msg_ctx_t *c, msg_stats_t *stats) {
  if (!c) return MSG_ERR_ARG;
  memset(c->t_ms, 0, sizeof(c->t_ms));
  return calc_numsol(c, stats);
}

int msg_gpu_advance(msg_ctx_t *c, int32_t nsteps, double rech_until, double rech_after, msg_run_stats_t *stats) {
  if (!c || nsteps < 0) return MSG_ERR_ARG;
  memset(c->t_ms, 0, sizeof(c->t_ms));
  cudaEventRecord(c->ev[5], c->stream);
  int rc = advance(c, nsteps, rech_until, rech_after, stats);
  cudaEventRecord(c->ev[6], c->stream);
  cudaEventSynchronize(c->ev[6]);
  float tot = 0.f;
  cudaEventElapsedTime(&tot, c->ev[5], c->ev[6]);
  c->t_ms[4] = tot;
  return rc;
}

// ---- restart file (checkpoint / resume) ------------------------------------------------
// The reference's restart file (write_rest, Nonlinear_solution.f90:792-816, and
// write_out_restf, Write_output.f90:415-432): gfortran sequential unformatted, two records
// -- real(DP) time, then head_new * len_scal for the ncalc cells -- each framed by a 4-byte
// record length before and after.  Records of 2^31 bytes or more (gfortran subrecords)
// are rejected.
static bool put_record(FILE *f, const void *p, size_t bytes) {
  const int32_t m = (int32_t)bytes;
  return fwrite(&m, 4, 1, f) == 1 && fwrite(p, 1, bytes, f) == bytes && fwrite(&m, 4, 1, f) == 1;
}

static bool get_record(FILE *f, void *p, size_t bytes) {
  int32_t m0 = 0, m1 = 0;
  return fread(&m0, 4, 1, f) == 1 && (size_t)m0 == bytes && fread(p, 1, bytes, f) == bytes &&
         fread(&m1, 4, 1, f) == 1 && m1 == m0;
}

int msg_gpu_write_restart(msg_ctx_t *c, const char *path) {
  if (!c || !path) return MSG_ERR_ARG;
  const size_t N = c->N;
  if (N * 8 > 0x7fffffffull) { set_error("write_restart: record of %zu bytes needs subrecords", N * 8); return MSG_ERR_SIZE; }
  std::vector<double> h(N);
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  MSG_CUDA(cudaMemcpy(h.data(), c->head_new, N * 8, cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < N; ++i) h[i] = h[i] * c->len_scal;
  const double t = c->current_t;   // already rounded to real(SP), as now_time is
  FILE *f = fopen(path, "wb");
  if (!f) { set_error("write_restart: cannot open %s", path); return MSG_ERR_ARG; }
  const bool ok = put_record(f, &t, 8) && put_record(f, h.data(), N * 8);
  if (fclose(f) != 0 || !ok) { set_error("write_restart: write failed on %s", path); return MSG_ERR_ARG; }
  return MSG_OK;
}

// assign_initv with a restart file (Assign_calculation.f90:416-434): time from record 1,
// heads = record 2 * (1 / len_scal).
int msg_gpu_read_restart(const char *path, int32_t ncalc, double len_scal, double *head, double *time) {
  if (!path || ncalc < 1 || !head || !(len_scal > 0.0)) return MSG_ERR_ARG;
  if ((size_t)ncalc * 8 > 0x7fffffffull) { set_error("read_restart: record needs subrecords"); return MSG_ERR_SIZE; }
  FILE *f = fopen(path, "rb");
  if (!f) { set_error("read_restart: cannot open %s", path); return MSG_ERR_ARG; }
  double t = 0.0;
  const bool ok = get_record(f, &t, 8) && get_record(f, head, (size_t)ncalc * 8);
  fclose(f);
  if (!ok) { set_error("read_restart: %s is not a restart file of %d cells", path, ncalc); return MSG_ERR_SIZE; }
  // assign_initv multiplies by len_scal_inv = SONE/len_scal, a real(SP) reciprocal
  // (Read_input.f90:1108, Assign_calculation.f90:433), and keeps the time as real(SP) (:431)
  const double inv = (double)(1.0f / (float)len_scal);
  for (int32_t i = 0; i < ncalc; ++i) head[i] = head[i] * inv;
  if (time) *time = (double)(float)t;
  return MSG_OK;
}

int msg_gpu_calc_mass(msg_ctx_t *c, double *out9) {
  if (!c || !out9) return MSG_ERR_ARG;
  double *d = nullptr;
  ALLOC(d, 9 * 8);
  int rc = launch_mass(c, d);
  if (rc) return rc;
  MSG_CUDA(cudaMemcpy(out9, d, 9 * 8, cudaMemcpyDeviceToHost));
  cudaFree(d);
  return MSG_OK;
}

int msg_gpu_cell_mass(msg_ctx_t *c, double *sto, double *con, double *sea, double *wel, double *rec, double *sur,
                      double *riv, double *lak, double *drn) {
  if (!c) return MSG_ERR_ARG;
  const size_t N = c->N, S = c->S;
  // Krylov scratch vectors (free between solves) hold the device copies: r, rs, v, p get
  // the [N] arrays; t holds the five [S] arrays back to back (N >= 5S needs nz >= 5, else
  // a temporary)
  double *ts = c->t;
  if ((size_t)N < 5 * S) ALLOC(ts, 5 * S * 8);
  int rc = launch_cell_mass(c, c->r, c->rs, c->v, c->p, ts, ts + S, ts + 2 * S, ts + 3 * S, ts + 4 * S);
  if (rc) { if (ts != c->t) cudaFree(ts); return rc; }
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  if (sto) MSG_CUDA(cudaMemcpy(sto, c->r, N * 8, cudaMemcpyDeviceToHost));
  if (con) MSG_CUDA(cudaMemcpy(con, c->rs, N * 8, cudaMemcpyDeviceToHost));
  if (sea) MSG_CUDA(cudaMemcpy(sea, c->v, N * 8, cudaMemcpyDeviceToHost));
  if (wel) MSG_CUDA(cudaMemcpy(wel, c->p, N * 8, cudaMemcpyDeviceToHost));
  double *hs[5] = {rec, sur, riv, lak, drn};
  for (int q = 0; q < 5; ++q)
    if (hs[q]) MSG_CUDA(cudaMemcpy(hs[q], ts + q * S, S * 8, cudaMemcpyDeviceToHost));
  if (ts != c->t) cudaFree(ts);
  return MSG_OK;
}

int msg_gpu_velocity(msg_ctx_t *c, double *facev, double *pointv) {
  if (!c) return MSG_ERR_ARG;
  const size_t N = c->N;
  double *dv = nullptr;
  ALLOC(dv, 9 * N * 8);
  int rc = launch_velocity(c, dv, dv + 6 * N);
  if (rc) { cudaFree(dv); return rc; }
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  if (facev) MSG_CUDA(cudaMemcpy(facev, dv, 6 * N * 8, cudaMemcpyDeviceToHost));
  if (pointv) MSG_CUDA(cudaMemcpy(pointv, dv + 6 * N, 3 * N * 8, cudaMemcpyDeviceToHost));
  cudaFree(dv);
  return MSG_OK;
}

int msg_gpu_set_wells(msg_ctx_t *c, int32_t nwell, const int32_t *well_index, const int32_t *well_conn,
                      const double *abyd_well, const double *well_bott, const double *read_well) {
  if (!c || nwell < 0) { set_error("set_wells: bad arguments"); return MSG_ERR_ARG; }
  int *wi = c->w_index, *wc = c->w_conn;
  double *wa = c->w_abyd, *wb = c->w_bott, *wr = c->w_rate;
  c->w_index = c->w_conn = nullptr; c->w_abyd = c->w_bott = c->w_rate = nullptr;
  c->nwell = 0;
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(wi); cudaFree(wc); cudaFree(wa); cudaFree(wb); cudaFree(wr);
  if (nwell == 0) {
    if (c->calc_well) MSG_CUDA(cudaMemsetAsync(c->calc_well, 0, (size_t)c->N * 8, c->stream));
    return MSG_OK;
  }
  if (!well_index || !well_conn || !abyd_well || !well_bott || !read_well) {
    set_error("set_wells: NULL array"); return MSG_ERR_ARG;
  }
  if (well_index[0] != 0) { set_error("set_wells: well_index[0] must be 0"); return MSG_ERR_ARG; }
  for (int w = 0; w < nwell; ++w)
    if (well_index[w + 1] < well_index[w]) { set_error("set_wells: well_index decreases at well %d", w + 1); return MSG_ERR_ARG; }
  const int nc = well_index[nwell];
  // a cell may belong to one well only (the reference accumulates calc_well from concurrent
  // threads, one per well); repeats within one well are added in order
  std::vector<int> owner(c->N, -1), conn0(nc);
  for (int w = 0; w < nwell; ++w)
    for (int k = well_index[w]; k < well_index[w + 1]; ++k) {
      int j = well_conn[k] - 1;
      if (j < 0 || j >= c->N) { set_error("set_wells: cell %d of well %d outside 1..%d", j + 1, w + 1, c->N); return MSG_ERR_ARG; }
      if (owner[j] >= 0 && owner[j] != w) {
        set_error("set_wells: cell %d belongs to wells %d and %d", j + 1, owner[j] + 1, w + 1); return MSG_ERR_ARG;
      }
      owner[j] = w;
      conn0[k] = j;
    }
  ALLOC(c->w_index, (size_t)(nwell + 1) * 4); ALLOC(c->w_conn, (size_t)std::max(nc, 1) * 4);
  ALLOC(c->w_abyd, (size_t)std::max(nc, 1) * 8); ALLOC(c->w_bott, (size_t)nwell * 8); ALLOC(c->w_rate, (size_t)nwell * 8);
  if (!c->calc_well) { ALLOC(c->calc_well, (size_t)c->N * 8); }
  MSG_CUDA(cudaMemsetAsync(c->calc_well, 0, (size_t)c->N * 8, c->stream));
  UPLOAD(c->w_index, well_index, (size_t)(nwell + 1) * 4);
  if (nc > 0) { UPLOAD(c->w_conn, conn0.data(), (size_t)nc * 4); UPLOAD(c->w_abyd, abyd_well, (size_t)nc * 8); }
  UPLOAD(c->w_bott, well_bott, (size_t)nwell * 8);
  UPLOAD(c->w_rate, read_well, (size_t)nwell * 8);
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  c->nwell = nwell;
  return MSG_OK;
}

// Dense [3S] stage / bed / area-by-distance table of the surface cells that carry a river
// (or lake); zeros elsewhere, which make the terms exact zeros.
static int set_stage(msg_ctx *c, double **dst, const char *what, int32_t n, const int32_t *cells, const double *head,
                     const double *bott, const double *abyd) {
  if (n < 0) { set_error("set_%s: n < 0", what); return MSG_ERR_ARG; }
  if (n == 0) {
    MSG_CUDA(cudaStreamSynchronize(c->stream));
    cudaFree(*dst); *dst = nullptr;
    return MSG_OK;
  }
  if (!cells || !head || !bott || !abyd) { set_error("set_%s: NULL array", what); return MSG_ERR_ARG; }
  const int S = c->S;
  std::vector<double> t((size_t)3 * S, 0.0);
  std::vector<char> seen(S, 0);
  for (int k = 0; k < n; ++k) {
    int s = cells[k] - 1;
    if (s < 0 || s >= S) { set_error("set_%s: surface cell %d outside 1..%d", what, s + 1, S); return MSG_ERR_ARG; }
    if (seen[s]) { set_error("set_%s: surface cell %d listed twice", what, s + 1); return MSG_ERR_ARG; }
    seen[s] = 1;
    t[s] = head[k]; t[(size_t)S + s] = bott[k]; t[(size_t)2 * S + s] = abyd[k];
  }
  if (!*dst) ALLOC(*dst, (size_t)3 * S * 8);
  UPLOAD(*dst, t.data(), (size_t)3 * S * 8);
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  return MSG_OK;
}

int msg_gpu_set_rivers(msg_ctx_t *c, int32_t n, const int32_t *rive2cals, const double *rive_head,
                       const double *rive_bott, const double *abyd_rive) {
  if (!c) return MSG_ERR_ARG;
  return set_stage(c, &c->riv, "rivers", n, rive2cals, rive_head, rive_bott, abyd_rive);
}

int msg_gpu_set_lakes(msg_ctx_t *c, int32_t n, const int32_t *lake2cals, const double *lake_head,
                      const double *lake_bott, const double *abyd_lake) {
  if (!c) return MSG_ERR_ARG;
  return set_stage(c, &c->lak, "lakes", n, lake2cals, lake_head, lake_bott, abyd_lake);
}

int msg_gpu_water_table(msg_ctx_t *c, double *wtable) {
  if (!c || !wtable) return MSG_ERR_ARG;
  int rc = launch_water_table(c, c->tmpv);   // tmpv: N >= S doubles of scratch
  if (rc) return rc;
  MSG_CUDA(cudaMemcpyAsync(wtable, c->tmpv, (size_t)c->S * 8, cudaMemcpyDeviceToHost, c->stream));
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  return MSG_OK;
}

int msg_gpu_set_convlog(msg_ctx_t *c, int32_t on) {
  if (!c) return MSG_ERR_ARG;
  if (on && !c->clog) c->clog = new (std::nothrow) ConvLog();
  if (on && !c->clog) { set_error("set_convlog: out of host memory"); return MSG_ERR_SIZE; }
  c->clog_on = on ? 1 : 0;
  return MSG_OK;
}

int msg_gpu_convlog(msg_ctx_t *c, msg_convrec_t *out, int32_t cap) {
  if (!c || cap < 0 || (cap > 0 && !out)) return MSG_ERR_ARG;
  if (!c->clog) return 0;
  ConvLog &q = *reinterpret_cast<ConvLog *>(c->clog);
  int k = 0;
  while (k < cap && !q.empty()) { out[k++] = q.front(); q.pop_front(); }
  return k;
}

int msg_gpu_timers(msg_ctx_t *c, double *ms5) {
  if (!c || !ms5) return MSG_ERR_ARG;
  for (int k = 0; k < 5; ++k) ms5[k] = c->t_ms[k];
  return MSG_OK;
}

long long msg_gpu_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

// Time `reps` back-to-back launches of one kernel class on the context's stream
// with CUDA events (the state of the last step is used as input):
// 0 = stencil SpMV (FP64 DIA), 1 = calc_func (vG pass + flux pass),
// 2 = make_matvec (vG pair + assembly), 3 = preconditioner apply, 4 = AMG setup,
// 5 = the four tensor-core convolutions of the learned guess (needs an attached network).
int msg_gpu_kernel_time(msg_ctx_t *c, int32_t which, int32_t reps, double *ms_per_launch) {
  if (!c || reps < 1 || !ms_per_launch) return MSG_ERR_ARG;
  int rc = MSG_OK;
  if (which == 3 && (c->prm.precon_type == 0 || c->prm.ref_quirks)) {
    if ((rc = launch_precon_dilu(c))) return rc;
  }
  if (which == 5) {
    if (!learned_ready(c) || c->timestep_num < 1) {
      set_error("kernel_time 5: no network attached or no previous time level");
      return MSG_ERR_STATE;
    }
    const float *o = nullptr;
    if ((rc = learned_forward(c, &o, nullptr, nullptr))) return rc;   // features into the padded buffer
  }
  auto one = [&]() -> int {
    switch (which) {
      case 0: return launch_spmv(c, c->head_new, c->tmpv);
      case 1: return launch_calc_func(c, c->head_new, c->new_f, false);
      case 2: return launch_make_matvec(c);
      case 3: return apply_prec(c, c->rhs, c->z);
      case 4: return (c->prm.precon_type == 1 && !c->prm.ref_quirks) ? amg_setup(c) : MSG_OK;
      case 5: return learned_convs(c);
      default: return MSG_ERR_ARG;
    }
  };
  if ((rc = one())) return rc;   // warm-up
  MSG_CUDA(cudaEventRecord(c->ev[5], c->stream));
  for (int k = 0; k < reps; ++k)
    if ((rc = one())) return rc;
  MSG_CUDA(cudaEventRecord(c->ev[6], c->stream));
  MSG_CUDA(cudaEventSynchronize(c->ev[6]));
  float ms = 0.f;
  MSG_CUDA(cudaEventElapsedTime(&ms, c->ev[5], c->ev[6]));
  *ms_per_launch = (double)ms / reps;
  if (which == 5) return learned_check(c);
  return MSG_OK;
}

int msg_gpu_set_tuning(msg_ctx_t *c, int32_t blk_cell, int32_t blk_smooth) {
  auto ok = [](int b) { return b >= 32 && b <= 1024 && (b % 32) == 0; };
  if (!c || !ok(blk_cell) || !ok(blk_smooth)) { set_error("set_tuning: block sizes must be multiples of 32 in 32..1024"); return MSG_ERR_ARG; }
  c->blk_cell = blk_cell;
  c->blk_smooth = blk_smooth;
  return MSG_OK;
}

// Ensemble driver: worker threads take members from a shared queue and advance each
// for nsteps accepted steps on the member's own stream, so members of uneven size and
// uneven Newton counts keep the GPU busy together.
int msg_gpu_ensemble_advance(msg_ctx_t **ctx, int32_t n, int32_t nsteps, const double *rech_until,
                             const double *rech_after, int32_t nworkers, msg_run_stats_t *stats) {
  if (!ctx || n < 1 || nsteps < 0 || nworkers < 1) return MSG_ERR_ARG;
  for (int k = 0; k < n; ++k) if (!ctx[k]) return MSG_ERR_ARG;
  int dev = 0;
  MSG_CUDA(cudaGetDevice(&dev));
  std::atomic<int> next(0), err(0);
  std::vector<std::string> msgs(n);
  auto work = [&]() {
    cudaSetDevice(dev);
    for (;;) {
      int k = next.fetch_add(1);
      if (k >= n) return;
      msg_run_stats_t st;
      memset(&st, 0, sizeof(st));
      int rc = advance(ctx[k], nsteps, rech_until ? rech_until[k] : 1.0e30, rech_after ? rech_after[k] : 1.0, &st);
      if (rc < 0) { err.store(rc); msgs[k] = get_error(); }
      if (stats) stats[k] = st;
    }
  };
  int nw = std::min<int>(nworkers, n);
  std::vector<std::thread> pool;
  for (int w = 0; w < nw; ++w) pool.emplace_back(work);
  for (auto &t : pool) t.join();
  if (err.load() < 0) {
    for (int k = 0; k < n; ++k)
      if (!msgs[k].empty()) { set_error("ensemble member %d: %s", k, msgs[k].c_str()); break; }
    return err.load();
  }
  return MSG_OK;
}

int msg_gpu_set_timing(msg_ctx_t *c, int32_t on) {
  if (!c) return MSG_ERR_ARG;
  c->timing = on;
  return MSG_OK;
}

}  // extern "C"

namespace msg {
static void free_ctx(msg_ctx *c) {
  if (c->stream) cudaStreamSynchronize(c->stream);
  delete reinterpret_cast<ConvLog *>(c->clog);
  c->clog = nullptr;
  amg_free(c);
  learned_free(c);
  void *dp[] = {c->reta, c->retn, c->resi, c->poro, c->ss, c->ksz, c->cell_top, c->cell_vol, c->hy, c->ab,
                c->invd, c->top_invd, c->w_index, c->w_conn, c->w_abyd, c->w_bott, c->w_rate, c->calc_well,
                c->riv, c->lak,
                c->surf_top, c->surf_bott, c->surf_reli, c->surf_parm, c->hydf_surf, c->abyd_surf, c->calc_rech,
                c->rech_base, c->sea_hydf, c->sea_abyd, c->read_seal, c->drain, c->offind, c->offrow, c->conn_dir,
                c->left_off, c->right_off, c->hydf_conn, c->abyd_conn, c->head_new, c->head_old, c->head_pre,
                c->head_change, c->srat_new, c->srat_old, c->surf_head, c->surf_old, c->new_f, c->kr, c->kr_per,
                c->alp, c->sto, c->stod, c->tmpv, c->dmat, c->lu, c->rhs, c->rhs_alt, c->head_old2, c->slope_rhs, c->dilu_d, c->r, c->rs,
                c->p, c->v, c->t, c->z, c->part, c->plane_ptr, c->plane_cells, c->dmat_f, c->lu_f, c->dres};
  for (auto q : dp) if (q) cudaFree(q);
  if (c->hpin) cudaFreeHost(c->hpin);
  for (int k = 0; k < 8; ++k) if (c->ev[k]) cudaEventDestroy(c->ev[k]);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}
}  // namespace msg
