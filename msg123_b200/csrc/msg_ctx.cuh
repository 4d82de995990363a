// msg_ctx.cuh -- device-side state of one solver context and the internal host API
// between the translation units of libmsg123gpu.so.
#pragma once
#include "msg_common.cuh"
#include "../../include/msg123_gpu.h"

namespace msg {

struct AmgLevel;   // msg_amg.cu

// Scalars of the Krylov / Newton recurrences kept in device memory.
struct DevScalars {
  double sk, sk0, sk2, alpha, beta, omega, ts, tt, rnorm, bnorm, errtol;
  int conv, in_iter, done, pad;
};

}  // namespace msg

struct msg_ctx {
  // ---- sizes --------------------------------------------------------------------
  int nx, ny, nz, N, S, nxy, nnz;
  int sea_top, free_drainage;
  msg_params_t prm;
  double len_scal, newper, newper_inv;
  double delt, delt_inv;
  int device;
  cudaStream_t stream;

  // ---- cell data (structured, reference local order) ------------------------------
  float *reta, *retn, *resi, *poro, *ss;        // [N] real(SP)
  double *cell_top, *cell_vol;                   // [N]
  double *hy, *ab;                               // [3N] hydf / abyd of the up, north, west face of each cell
  double *invd;                                  // [3N] 1/dis12 of the same faces (velocity output)
  double *top_invd;                              // [S] 1/dis2face(up) of each top cell (surface and sea faces)
  float *ksz;                                    // [N] kept for the drainage and surface coefficients
  // ---- surface (top layer) and boundary arrays [S] -----------------------------------
  double *surf_top, *surf_bott, *surf_reli, *surf_parm, *hydf_surf, *abyd_surf;
  double *calc_rech, *rech_base;
  double *sea_hydf, *sea_abyd, *read_seal;
  double *drain;                                 // [S] bottom-layer drainage coefficient
  // ---- wells, rivers, lakes (msg_gpu_set_wells / _rivers / _lakes; null when none) -----
  int nwell;
  int *w_index, *w_conn;                         // [nwell+1] prefix offsets, [nconn] 0-based cells
  double *w_abyd, *w_bott, *w_rate;              // per connection / per well / per well
  double *calc_well;                             // [N] well rates of the time step
  double *riv, *lak;                             // [3S] stage, bed, area/distance per surface cell
  // ---- reference CSR built on the GPU (export / tests) -------------------------------
  int *offind, *offrow, *conn_dir, *left_off, *right_off;
  double *hydf_conn, *abyd_conn;
  // ---- state -------------------------------------------------------------------------
  double *head_new, *head_old, *head_pre, *head_change, *srat_new, *srat_old, *head_old2;
  double *surf_head, *surf_old, *new_f;
  double *kr, *kr_per, *alp, *sto, *stod;        // per-cell vG results / storage terms
  double *tmpv;                                  // [N] spare vector (J.v, line search)
  // ---- level-1 system, DIA: lu[d*N + i] = J(i, nb_d(i)) --------------------------------
  double *dmat, *lu, *rhs, *slope_rhs;
  double *rhs_alt;                               // rhs assembled ahead by the line search (asm_ahead)
  float *dmat_f, *lu_f;                          // FP32 images (precision = 1)
  // ---- Krylov work ----------------------------------------------------------------------
  double *dilu_d, *r, *rs, *p, *v, *t, *z;
  msg::DevScalars *sc;                           // device scalars
  msg::DevScalars *sc_host;                      // pinned mirror
  double *part;                                  // reduction partials [npart]
  size_t npart;
  double *hpin;                                  // pinned host scalars
  double *dres;                                  // device reduction results [16]
  // ---- wavefront ordering for DILU --------------------------------------------------------
  int *plane_ptr, *plane_cells;
  int nplanes;
  // ---- AMG ----------------------------------------------------------------------------------
  void *amg;                                     // msg::AmgState (msg_amg.cu)
  int amg_nlevel, amg_age, amg_force;
  // ---- Newton module variables (Nonlinear_solution.f90:24-27) ---------------------------------
  int back_iter, back_flag, beta_iter, in_iter, conv_flag, out_iter;
  double maxvar, l2_new, l2_pre, l2_jnorm, lam, eta, gradient, maxstep, errtol, bnorm, rnorm;
  double l2_last;    // squared norm of the last residual evaluated through func_norm
  // ---- time loop ---------------------------------------------------------------------------------
  double current_t, delt_old1, delt_old2;
  int timestep_num, last_conv, last_out;
  int guess_fallbacks;                           // learned guesses replaced by extrapolation
  int guess_rejected;                            // learned guesses not used (larger residual)
  int guess_skip, guess_backoff;                 // guess_select 2: steps left without the network, next pause
  int vg_at_head;                                // S, kr, storage in memory are those of head_new (reuse)
  int asm_ahead;                                 // dmat, lu, rhs_alt: the system assembled at head_new
  int head_moved;                                // the line search moved head_new off the full step
  // convergence log (msg_gpu_set_convlog): records of the Newton iterations, oldest first
  void *clog;                                    // std::deque<msg_convrec_t> (msg_api.cu)
  int clog_on;
  // learned initial guess (msg_learned.cu)
  void *learned;
  // ---- timing ------------------------------------------------------------------------------------
  cudaEvent_t ev[8];
  double t_ms[5];
  int timing;
  // ---- launch shapes chosen by the autotuner (kernels without reductions only) ---------------
  int blk_cell;      // block size of the van Genuchten / storage pass (k_cell)
  int blk_smooth;    // block size of the level-1 Jacobi / residual passes of the V-cycle
};

namespace msg {

// ---- msg_physics.cu ---------------------------------------------------------------------------
int build_connectivity(msg_ctx *c, const msg_grid_t *g);
int launch_srat_rperm(msg_ctx *c, const double *h, double pertur, double *srat, double *kr, double *alp);
int launch_water_table(msg_ctx *c, double *wt);
// F = calc_func(h); also writes srat_new and kr (rel_perm).  partial sums of F^2 in c->part[0..].
int launch_calc_func(msg_ctx *c, const double *h, double *F, bool norm);
// make_matvec at c->head_new: dmat, lu (DIA), rhs = -F.  reuse: srat_new, kr and sto
// already hold the values at head_new (the last calc_func was evaluated there).
int launch_make_matvec(msg_ctx *c, bool reuse = false, double *rhs_out = nullptr);   // rhs_out null: c->rhs
// Export the DIA Jacobian into the reference CSR order.
int launch_dia_to_csr(msg_ctx *c, double *lumat_dev);
int launch_mass(msg_ctx *c, double *out9_dev);
int launch_velocity(msg_ctx *c, double *facev, double *pointv);
int launch_cell_mass(msg_ctx *c, double *sto, double *con, double *sea, double *wel, double *rec, double *sur,
                     double *riv, double *lak, double *drn);
int launch_wells(msg_ctx *c);
int flux_parts(const msg_ctx *c);   // F^2 partials the assembly pass writes (one per block)

// ---- msg_linear.cu ----------------------------------------------------------------------------
int build_wavefront(msg_ctx *c);
int launch_precon_dilu(msg_ctx *c);
int launch_solve_ilu(msg_ctx *c, const double *b, double *x);
int launch_spmv(msg_ctx *c, const double *x, double *y);
// x in/out (device), uses c->rhs, c->bnorm, c->errtol; x_zero: x holds zeros on entry
int solve_bicgs(msg_ctx *c, double *x, bool x_zero = false);
// reductions (results land in c->hpin after a sync)
int dot(msg_ctx *c, const double *a, const double *b, int n, double *out);   // sync + host value
// sum narr partial arrays (nparts each, consecutive in c->part) on the device; sync; host values
int finish(msg_ctx *c, int nparts, int narr, double *out);
int finish_to(msg_ctx *c, int nparts, int narr, int slot);   // into dres[slot..], no wait
int fetch_res(msg_ctx *c, int count, double *out);           // dres[0..count) to the host (waits)
int norm1(msg_ctx *c, const double *a, int n, double *out);
int abserrmax(msg_ctx *c, double *xn, const double *xp, double *chmax, double *xmax, int *nun, int *nan,
              const double *dh = nullptr);   // dh: form xn = xp + dh first
int lam_length(msg_ctx *c, const double *dh, const double *hn, double *out);
// ||dh||^2, ||f||^2, (s, jv) (jv null: (s, b - r)) and lam_length(dh, hn) in one pass
int backtr_stats(msg_ctx *c, const double *dh, const double *hn, const double *f, const double *s, const double *jv,
                 const double *b, const double *r, double out[5], bool slot4);   // slot4: also dres[4] (pending)
int axpby(msg_ctx *c, double *y, const double *x, double a, const double *w, int n);   // y = x + a*w
int scale(msg_ctx *c, double *y, double a, int n);

// ---- msg_amg.cu ---------------------------------------------------------------------------------
int amg_setup(msg_ctx *c);
int amg_reserve(msg_ctx *c);   // the hierarchy's device arena, reserved when the context is made
int amg_apply(msg_ctx *c, const double *r, double *z);
void amg_free(msg_ctx *c);

// ---- msg_learned.cu ------------------------------------------------------------------------------
bool learned_ready(msg_ctx *c);
int learned_guess(msg_ctx *c);
// features + tensor-core forward pass of the attached network (no state change)
int learned_forward(msg_ctx *c, const float **out, double *s_out, double *ratio_out);
// the four convolutions again on the features of the last learned_forward (timing)
int learned_convs(msg_ctx *c);
int learned_check(msg_ctx *c);   // sync + status of the last tensor-core pass
void learned_free(msg_ctx *c);

// ---- preconditioner dispatch (msg_linear.cu) ---------------------------------------------------------
int apply_prec(msg_ctx *c, const double *r, double *z);

// ---- scan (msg_linear.cu) ---------------------------------------------------------------------------
int scan_exclusive(msg_ctx *c, const int *in, int *out, int n, int *total_host);

}  // namespace msg
