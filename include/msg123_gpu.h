/*
 * msg123_gpu.h -- C ABI of the B200 Newton-Krylov library for the 3D Richards
 * equation (drop-in for Msg123's Nonlinear_solution / Linear_solution path).
 *
 * All entry points take plain host pointers and sizes.  The library copies the
 * inputs to device memory, owns every device allocation, and returns an int
 * status: 0 = ok, >0 = soft failure (no convergence), <0 = hard error (message
 * in msg_gpu_last_error()).  No exception ever crosses the ABI.  One context
 * per host thread.
 *
 * Units follow the reference after nondimensionalisation: every length is
 * divided by len_scal (reference Read_input.f90:1100-1112), alpha and Ss are
 * multiplied by it and Ks is divided by it (Assign_calculation.f90:117,259-260).
 * Cell numbering is the reference local order: x fastest, then y, then layers
 * from the top down (Set_cell.f90:845-925).  Face order is
 * up(1) north(2) west(3) east(4) south(5) down(6) (Set_condition.f90:1584-2026).
 */
#ifndef MSG123_GPU_H
#define MSG123_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define MSG_API __attribute__((visibility("default")))
#else
#define MSG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (Newton / Krylov / time loop outcome). */
enum {
  MSG_OK = 0,
  MSG_NEWTON_MAXIT = 1,      /* out_iter reached maxout_iter      (Nonlinear_solution.f90:278-282) */
  MSG_NAN = 2,               /* NaN in the update                  (Nonlinear_solution.f90:151-155) */
  MSG_LINESEARCH_FAIL = 3,   /* back_flag set by run_backtr        (Nonlinear_solution.f90:265-269) */
  MSG_DIVERGED = 4,          /* |dh| >= VARMAX or |h| >= XMAX       (Nonlinear_solution.f90:283-287) */
  MSG_DT_TOO_SMALL = 5,      /* delt < DSMAL                        (Time_module.f90:72-73) */
  MSG_ERR_ARG = -1,
  MSG_ERR_CUDA = -2,
  MSG_ERR_SIZE = -3,
  MSG_ERR_STATE = -4
};

/* Problem description: what set_cell_info / make_cell / set_connect consume.
 * Arrays are host pointers, read only during msg_gpu_create. */
typedef struct msg_grid {
  int32_t nx, ny, nz;        /* active box; ncalc = nx*ny*nz, ncals = nx*ny (top layer) */
  int32_t sea_top;           /* 1: a fixed-head ("sea") layer sits above the top layer   */
  int32_t free_drainage;     /* 1: unit-gradient outflow through the bottom face (extension, no reference counterpart) */
  int32_t pad0;
  const float *reta, *retn, *resi, *poro, *ss;  /* [ncalc] real(SP) soil parameters (Assign_calculation.f90:19-21) */
  const float *ksx, *ksy, *ksz;                  /* [ncalc] real(SP) saturated conductivity                */
  const double *cell_top, *cell_vol;             /* [ncalc] (Make_cell.f90:11-13)                          */
  const double *dis2face;    /* [6*ncalc] centre-to-face distance, face-major: [f*ncalc + i]               */
  const double *face_area;   /* [6*ncalc] face areas, face-major                                           */
  const double *area_r;      /* [ncals] plan area that receives recharge (rech_area)                       */
  const double *surf_top, *surf_bott, *surf_reli, *surf_parm;  /* [ncals] surface term (Prep_calculation.f90:173-201) */
  const double *sea_head;    /* [ncals] fixed head of the sea cell above each top cell (read_seal)          */
} msg_grid_t;

/* Solver knobs: the namelist set_solution / set_amg (Initial_module.f90:355-359)
 * plus the extensions the synthetic configurations need. */
typedef struct msg_params {
  double len_scal;           /* real(SP) len_scal promoted to double                                 */
  double criteria;           /* Newton criterion on max|dh|*len_scal (Nonlinear_solution.f90:144-150) */
  double lin_tol;            /* >0: fixed BiCGStab tolerance; 0: Eisenstat-Walker eta (reference)     */
  int32_t criteria_rel;      /* 1: criteria is multiplied by max|h|*len_scal (relative head tolerance) */
  int32_t maxout_iter;       /* Newton iteration cap                                                  */
  int32_t maxinn_iter;       /* BiCGStab iteration cap                                                */
  int32_t precon_type;       /* 0: DILU / ILU(0); 1: AMG                                              */
  int32_t ref_quirks;        /* 1: AMG preconditioner reproduces the reference (output = fine DILU)    */
  int32_t precision;         /* 0: FP64 everywhere; 1: FP32 V-cycle, BF16 coarse operators            */
  int32_t amg_nlevel;        /* maximum number of AMG levels                                          */
  int32_t amg_coarse_max;    /* coarsest level is solved directly once it has <= this many rows       */
  int32_t amg_sweeps;        /* Jacobi sweeps before and after the coarse correction                  */
  float jac_omega;           /* prolongation smoothing weight (real(SP))                               */
  float amg_theta;           /* strength threshold (real(SP))                                          */
  float smooth_omega;        /* Jacobi smoother weight                                                */
  int32_t sim_type;          /* 0: delt*inc_fact per accepted step; 1: heuristic (apply_heuri)         */
  int32_t amg_lag;           /* 0: AMG rebuilt at every make_matvec (reference); k >= 1: rebuilt at the
                                first Newton iteration of every k-th time step                         */
  double ini_step;           /* initial delt (s)                                                      */
  double inc_fact;           /* factor for sim_type 0                                                 */
  double max_step;           /* cap on delt for sim_type 1                                            */
  double end_time;           /* simulation end (s)                                                    */
  int32_t guess_mode;        /* Newton initial guess: 0 = previous head (reference), 1 = linear
                                extrapolation, 2 = learned increment                                  */
  int32_t guess_select;      /* guess_mode 2: 1 = start from whichever of the learned and the
                                extrapolated guess has the smaller ||F|| (two residual evaluations;
                                when the extrapolation wins, the first assembly reuses its van
                                Genuchten state); 2 = as 1, and after the extrapolation wins the
                                network pauses for 1, 2, 4, then 8 steps (reset when it wins);
                                a failed solve from the learned guess is redone from the
                                extrapolation when the guess was not vetted (0) or Newton broke
                                down (NaN, divergence), else the step is rejected as usual          */
  int32_t vg_form;           /* Mualem kr: 0 = the reference's expression (four pow per cell);
                                1 = the same function with Se^(1/m) = 1/(1+beta) and
                                beta^m = (alpha|h|)^(n-1): two pow per cell; differs from 0 by
                                rounding only                                                     */
  int32_t jv_mode;           /* J.dh of the line-search slope: 0 = Brown-Saad differencing of F
                                (calc_vecjacf, the reference: one more residual evaluation per
                                Newton iteration); 1 = rhs - r, the assembled Jacobian times dh as
                                BiCGStab's own residual r leaves it (ref_quirks = 0 only)          */
} msg_params_t;

/* Per-Newton-solve statistics (fields of the reference conv log, Nonlinear_solution.f90:59-63). */
typedef struct msg_stats {
  int32_t status;            /* MSG_OK when converged                                 */
  int32_t out_iter;          /* Newton iterations                                     */
  int32_t inner_total;       /* BiCGStab iterations summed over the Newton iterations */
  int32_t back_total;        /* backtracking steps summed                             */
  int32_t in_iter_last, back_iter_last;
  int32_t maxnun;            /* 1-based cell of the largest change (last iteration)   */
  int32_t pad;
  double maxvar;             /* signed largest change * len_scal                      */
  double l2_new;             /* ||F(h)||^2 at exit                                    */
} msg_stats_t;

/* Time loop statistics. */
typedef struct msg_run_stats {
  int32_t status;
  int32_t accepted;          /* accepted time steps                      */
  int32_t rejected;          /* rejected attempts (dt halved)             */
  int32_t newton_total;      /* Newton iterations over accepted + rejected */
  int32_t krylov_total;
  int32_t back_total;
  double current_t;          /* simulated time reached (s)               */
  double delt;               /* delt after the last step                  */
} msg_run_stats_t;

/* One Newton iteration, as a line of the reference's convergence log (written inside
   calc_numsol, Nonlinear_solution.f90:59-63,240-252).  Scaled as the reference prints them. */
typedef struct msg_convrec {
  double time;               /* current time of the step being solved (s)                       */
  double delt;               /* its time step (s)                                               */
  int32_t out_iter;          /* OUTER                                                           */
  int32_t in_iter;           /* INNER: Krylov iterations of this Newton iteration               */
  int32_t back_iter;         /* BACK: line-search backtracks                                    */
  int32_t cell;              /* 1-based local cell number of the largest change (maxnun)        */
  double maxvar;             /* MAXIMUM CHANGE: signed largest head change * len_scal           */
  double dmat;               /* DIAGONAL MATRIX at that cell * len_scal^2                       */
  double rhs;                /* RIGHT HAND VECTOR at that cell * len_scal^3                     */
  double head;               /* UNKNOWN VALUE: head at that cell * len_scal                     */
  int32_t status;            /* -1: the solve went on; else the solve's status (MSG_OK, ...)    */
  int32_t pad;
} msg_convrec_t;

typedef struct msg_ctx msg_ctx_t;

/* Last error message of this thread. */
MSG_API const char *msg_gpu_last_error(void);

/* Allocate a context on the current CUDA device and build the connectivity on
 * the GPU.  Replaces allocate_solvar + set_connect (Allocate_solution.f90:56-197,
 * Set_condition.f90:1584-2158) and prepare_calc's newper (Prep_calculation.f90:79). */
MSG_API int msg_gpu_create(const msg_grid_t *grid, const msg_params_t *params, msg_ctx_t **out);
MSG_API void msg_gpu_destroy(msg_ctx_t *ctx);

/* Export the reference CSR built on the GPU (off_index, off_row 1-based, conn_dir,
 * left_off, right_off, sat_hydf, area_dis; Set_condition.f90:1584-2026).  Each
 * pointer may be NULL.  nnz receives off_index(ncalc). */
MSG_API int msg_gpu_get_connect(msg_ctx_t *ctx, int32_t *offind, int32_t *offrow, int32_t *conn_dir,
                        int32_t *left_off, int32_t *right_off, double *hydf_conn,
                        double *abyd_conn, int32_t *nnz);

/* Set the time-level state and delt.  NULL (or delt <= 0) leaves a field unchanged.
 * surf_head sets BOTH the surface head and surf_old, the surface head a rejected step
 * rolls back to (Time_module.f90:253-264): a host that passes surf_head in the middle
 * of a step therefore also moves that rollback point.  A host that restores a saved
 * state between steps passes the surf_head it read with msg_gpu_get_state, which is
 * then the rollback point of the next step as in the reference. */
MSG_API int msg_gpu_set_state(msg_ctx_t *ctx, const double *head_new, const double *head_old,
                      const double *srat_old, const double *surf_head, double delt);
/* Copy the whole time level of src into dst, two contexts of the same grid on the same
 * device: heads and saturations of both time levels, the level before them (the linear
 * extrapolation and the learned guess read it), surface heads, recharge, the clock, delt
 * and the step history apply_heuri and the guesses use.  Solver settings, the AMG
 * hierarchy (rebuilt at dst's next Newton iteration) and the counters stay dst's own.
 * So several settings can advance from one state, e.g. to compare them over the same
 * window.  No counterpart in the reference, whose time level lives in module globals. */
MSG_API int msg_gpu_copy_state(msg_ctx_t *dst, const msg_ctx_t *src);
MSG_API int msg_gpu_get_state(msg_ctx_t *ctx, double *head_new, double *head_old, double *srat_new,
                      double *srat_old, double *surf_head);

/* t = 0 branch of calc_nextst (Time_module.f90:142-196): head_new = head_old = head,
 * srat_old = srat_new = calc_srat_rperm(head), surf_head = surf_old = head (top layer). */
MSG_API int msg_gpu_init_state(msg_ctx_t *ctx, const double *head, double delt);

/* Recharge volume rate per surface cell (calc_rech, Time_module.f90:88-94). */
MSG_API int msg_gpu_set_recharge(msg_ctx_t *ctx, const double *calc_rech);

/* calc_srat_rperm (Calc_parameter.f90:15-77) on a host head vector. */
MSG_API int msg_gpu_srat_rperm(msg_ctx_t *ctx, const double *pres, double pertur, double *srat,
                       double *rperm, double *sstor);

/* calc_func (Calc_function.f90:24-101): funcv = F(infx). */
MSG_API int msg_gpu_calc_func(msg_ctx_t *ctx, const double *infx, double *funcv);

/* make_matvec (Make_linearsystem.f90:24-68) at the current head_new: the Jacobian
 * diagonal dmat[ncalc], off-diagonals lumat[nnz] in the reference CSR order and
 * rhs = -F.  Any output may be NULL; the system stays on the device for the
 * next msg_gpu_solve_linalg. */
MSG_API int msg_gpu_make_matvec(msg_ctx_t *ctx, double *dmat, double *lumat, double *rhs);

/* Load a level-1 system array_var(1)%{dmat,lumat,rhs} (lumat in reference CSR order)
 * as make_matvec would leave it, and build the AMG hierarchy when precon_type = 1. */
MSG_API int msg_gpu_set_system(msg_ctx_t *ctx, const double *dmat, const double *lumat, const double *rhs);

/* Apply the preconditioner of the current system once: z = M^-1 r (solve_ilu with the
 * DILU diagonal, Linear_solution.f90:742-855, or one AMG V-cycle). */
MSG_API int msg_gpu_precond(msg_ctx_t *ctx, const double *r, double *z);

/* calc_vecjacf (Calc_function.f90:515-621): out = J(x) v by Brown-Saad differencing. */
MSG_API int msg_gpu_vecjacf(msg_ctx_t *ctx, const double *x, const double *v, double *out);

/* solve_linalg (Linear_solution.f90:26-58): BiCGStab on the system of the last
 * make_matvec with bnorm = init_norm and tolerance errtol, starting from inx. */
MSG_API int msg_gpu_solve_linalg(msg_ctx_t *ctx, double init_norm, double errtol, double *inx,
                         double *last_norm, int32_t *in_iter, int32_t *conv_flag);

/* calc_numsol (Nonlinear_solution.f90:33-294): one time level's Newton solve.  Heads,
 * statistics and the convergence log are those of the reference's loop.  Unless the
 * convergence log, the phase timers or ref_quirks are on, the line search's residual
 * evaluation at the full step is an assembly (used by the next Newton iteration), so on
 * return the device's level-1 system may be the one assembled at the final head rather
 * than at the last iteration's; msg_gpu_make_matvec re-assembles it at head_new. */
MSG_API int msg_gpu_calc_numsol(msg_ctx_t *ctx, msg_stats_t *stats);

/* Time loop (Msg.f90:83-104 with update_tstep/calc_nextst, Time_module.f90:34-273):
 * advance until nsteps more steps are accepted or end_time is reached.
 * rech_until/rech_after: the recharge array applies until simulated time
 * rech_until (s), after which it is scaled by rech_after (0 = rain stops). */
MSG_API int msg_gpu_advance(msg_ctx_t *ctx, int32_t nsteps, double rech_until, double rech_after,
                    msg_run_stats_t *stats);

/* Wells, rivers and lakes (the reference's well / river / lake boundary terms).  Each call
 * replaces the table; n = 0 removes it.  Cells are 1-based as the reference stores them.
 *
 * msg_gpu_set_wells: the well connectivity set_wellconn builds -- well_index [nwell+1]
 * prefix offsets (well_index[0] = 0), well_conn [well_index[nwell]] cells, abyd_well per
 * connection -- and per well its bottom well_bott and pumping volume rate read_well.  At
 * the start of every time step after an accepted one (and of the first), msg_gpu_advance
 * sets the per-cell rates as set_vwell_head does (Time_module.f90:1137-1158 with
 * calc_vheadout / calc_vheadin, :1253-1335); calc_func adds them as func_wellterm does
 * (Calc_function.f90:277-302), with no Jacobian entry, as in make_matrix.  A cell may belong
 * to one well only.
 *
 * msg_gpu_set_rivers / msg_gpu_set_lakes: rive2cals / lake2cals (top-layer cells, each at
 * most once), stage, bed elevation and area/distance abyd_rive / abyd_lake of each river or
 * lake cell: func_riveterm / func_laketerm (Calc_function.f90:393-473) in the residual and
 * set_rivebound / set_lakebound (Make_linearsystem.f90:287-408) in the Jacobian diagonal.
 * Call again whenever the stages change (the reference's time series). */
MSG_API int msg_gpu_set_wells(msg_ctx_t *ctx, int32_t nwell, const int32_t *well_index, const int32_t *well_conn,
                              const double *abyd_well, const double *well_bott, const double *read_well);
MSG_API int msg_gpu_set_rivers(msg_ctx_t *ctx, int32_t n, const int32_t *rive2cals, const double *rive_head,
                               const double *rive_bott, const double *abyd_rive);
MSG_API int msg_gpu_set_lakes(msg_ctx_t *ctx, int32_t n, const int32_t *lake2cals, const double *lake_head,
                              const double *lake_bott, const double *abyd_lake);

/* calc_mass (Calc_function.f90:103-174) summed over cells: out[0..7] =
 * storage, flow, recharge, well, surface, river, lake, sea (+ out[8] drainage),
 * each a volume over the step (rate * delt). */
MSG_API int msg_gpu_calc_mass(msg_ctx_t *ctx, double *out9);
/* calc_cell_mas (Calc_output.f90:54-91, through calc_mass with sfla = 0): the step's
 * volumes per cell, in the arrays the reference adds into st_msloc for every regional
 * mass-balance output.  sto, con, sea, wel: [ncalc] (storage change, flow from the
 * neighbours, sea-face inflow, wells); rec, sur, riv, lak: [ncals] (recharge, surface,
 * river, lake); drn: [ncals] outflow through the bottom face of each column under free
 * drainage (extension, no reference column).  Each a rate times delt, summing to the
 * msg_gpu_calc_mass totals.  Any pointer may be NULL. */
MSG_API int msg_gpu_cell_mass(msg_ctx_t *ctx, double *sto, double *con, double *sea, double *wel, double *rec,
                              double *sur, double *riv, double *lak, double *drn);
/* calc_outvelc (Calc_output.f90:168-241) at the current head_new (relative permeability
 * recomputed there): facev [6*ncalc], face-major (facev[d*ncalc + i], d = up, north, west,
 * east, south, down), the Darcy velocity through each face, positive into the cell,
 * nondimensional like the reference's; pointv [3*ncalc] (x, y, z components, upward z
 * positive), the cell-centred velocity the reference writes.  Faces with no connection are
 * 0; under free drainage (extension) the bottom face of the lowest layer carries the
 * unit-gradient outflow -Ksz*kr.  Either pointer may be NULL. */
MSG_API int msg_gpu_velocity(msg_ctx_t *ctx, double *facev, double *pointv);
/* Water table of the current state (calc_wtable, Calc_output.f90:20-52, called by
 * write_out_wtabf with head_new and srat_new): for each surface column, the head of the
 * lowest cell that is not fully saturated (srat != 1), scanning up from the bottom layer;
 * the top cell's head when the whole column is saturated.  wtable: [ncals] host doubles,
 * nondimensional like head (the reference writes wtable * len_scal). */
MSG_API int msg_gpu_water_table(msg_ctx_t *ctx, double *wtable);
/* Restart file in the reference's format (replaces write_rest, Nonlinear_solution.f90:792-816,
   and write_out_restf, Write_output.f90:415-432): gfortran sequential unformatted records
   [real(DP) time][head_new * len_scal, ncalc values], 4-byte length markers. */
MSG_API int msg_gpu_write_restart(msg_ctx_t *ctx, const char *path);
/* Reads such a file (replaces the restart branch of assign_initv, Assign_calculation.f90:416-434):
   head = value * len_scal_inv with len_scal_inv = 1/len_scal rounded to single precision (as
   Read_input.f90:1108 forms it), time rounded to single precision; host code only, no GPU. */
MSG_API int msg_gpu_read_restart(const char *path, int32_t ncalc, double len_scal, double *head, double *time);

/* Device time spent in the last advance/numsol call split by phase (ms):
 * [0] assembly, [1] Krylov, [2] AMG setup, [3] residual evaluations, [4] total. */
MSG_API int msg_gpu_timers(msg_ctx_t *ctx, double *ms5);
/* Convergence log: with on = 1 every Newton iteration of calc_numsol / advance appends one
   msg_convrec_t to a buffer held by the context (three 8-byte device reads per iteration).
   msg_gpu_convlog moves up to `cap` records, oldest first, into `out` and returns how many
   (>= 0); the buffer keeps at most 2^20 records and drops the oldest beyond that. */
MSG_API int msg_gpu_set_convlog(msg_ctx_t *ctx, int32_t on);
MSG_API int msg_gpu_convlog(msg_ctx_t *ctx, msg_convrec_t *out, int32_t cap);
/* Time `reps` back-to-back launches of one kernel class on the context's stream with
 * CUDA events, inputs = the current state: 0 = stencil SpMV (FP64), 1 = calc_func,
 * 2 = make_matvec, 3 = one preconditioner apply, 4 = AMG setup, 5 = the four tensor-core
 * convolutions of the learned guess (needs an attached network and one accepted step).
 * Result in ms per launch. */
MSG_API int msg_gpu_kernel_time(msg_ctx_t *ctx, int32_t which, int32_t reps, double *ms_per_launch);

/* AMG hierarchy of the last setup (structural tests): level 0 is the Jacobian in CSR
 * form; level l > 0 holds its operator (off-diagonals CSR, 0-based columns, diagonal
 * apart as in array_var(l)%{dmat,lumat}), the prolongation P from it to level l-1 and
 * the aggregate of every level l-1 row (-1: none).  No counterpart returns these in
 * the reference; they mirror pro_var / crs_index / array_var (Allocate_solution.f90:22-50). */
MSG_API int msg_gpu_amg_nlevel(msg_ctx_t *ctx);
MSG_API int msg_gpu_amg_level_sizes(msg_ctx_t *ctx, int32_t lv, int32_t *n, int32_t *nnz, int32_t *pnnz);
MSG_API int msg_gpu_amg_level(msg_ctx_t *ctx, int32_t lv, int32_t *offind, int32_t *offrow, double *dmat,
                              double *lumat, int32_t *pindex, int32_t *poffrow, double *pval, int32_t *agg);

/* Dense FP64 inverse by Gauss-Jordan with partial pivoting (ties to the lowest row):
 * the coarsest-level solve of the AMG V-cycle (the reference's coarsest level is
 * smoothed by solve_ilu instead, Linear_solution.f90:617-660).  a and inv are host
 * arrays, row-major n x n.  Allocates its device buffers. */
MSG_API int msg_gpu_dense_inverse(int32_t n, const double *a, double *inv);

/* Allocation-free variant of msg_gpu_dense_inverse, for callers that cannot call
 * cudaMalloc (a host that passes device arrays it already owns, or a step running
 * under a fixed device-memory budget).  No counterpart exists in the reference.
 * a_dev / inv_dev: caller-owned device arrays, row-major n x n, 1 <= n <= 512 (larger n
 * returns MSG_ERR_SIZE).  Work is queued on `stream` (NULL: legacy default stream).
 * The workspace is one static device array per GPU (about 4 MiB, held until exit).
 * Every call looks up its address for the current device (so a cudaDeviceReset between
 * calls is safe); the first call on a device also loads the library's device code there
 * and should precede any stream capture.  Concurrent calls on one device race on that
 * workspace.  A singular input is not detected: its zero pivot gives inf/NaN entries
 * and the call still returns MSG_OK. */
MSG_API int msg_gpu_dense_inverse_noalloc(int32_t n, const double *a_dev, double *inv_dev, void *stream);

/* ---- learned Newton initial guess (no counterpart in the reference) ----------------------
 * A 3D CNN (four 3x3x3 convolutions, 16 channels, GELU, BF16 weights and activations,
 * FP32 accumulation on the tensor cores) predicts the correction to the linear
 * extrapolation of the head: h0 = h_t + r (h_t - h_{t-1}) + s * CNN(features).
 * Used by calc_numsol's time loop when guess_mode = 2; a step whose Newton solve fails
 * from the learned guess is retried from the plain extrapolation. */
typedef struct msg_cnn msg_cnn_t;
MSG_API int msg_gpu_cnn_create(int32_t seed, msg_cnn_t **out);
MSG_API void msg_gpu_cnn_destroy(msg_cnn_t *cnn);
MSG_API int msg_gpu_cnn_nparam(void);
/* corrections whose normalised size |o| is at most `dead` are dropped (default 0.1) */
MSG_API int msg_gpu_cnn_set_deadband(msg_cnn_t *cnn, float dead);
MSG_API int msg_gpu_cnn_get_weights(msg_cnn_t *cnn, float *w);
MSG_API int msg_gpu_cnn_set_weights(msg_cnn_t *cnn, const float *w);
/* append a training sample from a context right after an accepted step */
MSG_API int msg_gpu_cnn_collect(msg_cnn_t *cnn, msg_ctx_t *ctx);
MSG_API int msg_gpu_cnn_nsamples(msg_cnn_t *cnn);
/* bound the sample store to cap samples (0: unbounded): once full, each collected step
   replaces a uniformly drawn stored sample with probability cap / (steps collected), so the
   store stays a uniform sample of every step seen (reservoir sampling; seed seeds the draws) */
MSG_API int msg_gpu_cnn_set_capacity(msg_cnn_t *cnn, int32_t cap, int32_t seed);
/* steps offered to msg_gpu_cnn_collect since the capacity was set */
MSG_API long long msg_gpu_cnn_seen(msg_cnn_t *cnn);
/* append a sample from host arrays: x [N][16] features, y [N] target, N = nx*ny*nz */
MSG_API int msg_gpu_cnn_add_sample(msg_cnn_t *cnn, int32_t nx, int32_t ny, int32_t nz, const float *x, const float *y);
/* inference pass of the tensor-core (tcgen05) path on a stored sample; out: N floats.
   No reference counterpart (the learned guess is an addition of this library). */
MSG_API int msg_gpu_cnn_infer(msg_cnn_t *cnn, int32_t sample, float *out);
/* test hook for the bounded waits: as msg_gpu_cnn_infer, but the first convolution never
   loads the input box of tile `tile`; the kernel's wait on it runs out (about 1 s), the
   pass ends normally and the call returns MSG_ERR_CUDA with the wait's code in
   msg_gpu_last_error().  No reference counterpart. */
MSG_API int msg_gpu_cnn_infer_withhold(msg_cnn_t *cnn, int32_t sample, int32_t tile, float *out);
/* mean squared error on one sample; grad (msg_gpu_cnn_nparam floats) and out (N) may be NULL */
MSG_API int msg_gpu_cnn_loss_grad(msg_cnn_t *cnn, int32_t sample, double *loss, float *grad, float *out);
/* AdamW training over the stored samples */
MSG_API int msg_gpu_cnn_train(msg_cnn_t *cnn, int32_t iters, float lr, float weight_decay, int32_t seed,
                              double *mean_loss);
/* use the network in a context (guess_mode = 2); NULL detaches.  One network may serve
   several contexts, also from several host threads: their guesses take turns on it.  Do
   not change or train its weights while attached contexts advance. */
MSG_API int msg_gpu_cnn_attach(msg_ctx_t *ctx, msg_cnn_t *cnn);
/* learned guesses replaced by the extrapolation after a failed Newton solve */
MSG_API int msg_gpu_guess_fallbacks(msg_ctx_t *ctx);
/* learned guesses not used because the extrapolation had the smaller residual */
MSG_API int msg_gpu_guess_rejected(msg_ctx_t *ctx);

/* Number of kernels this library has launched in this process (all contexts). */
MSG_API long long msg_gpu_launch_count(void);

/* Launch shapes for the kernels without reductions (multiples of 32 in 32..1024):
 * blk_cell for the van Genuchten/storage pass, blk_smooth for the level-1 Jacobi and
 * residual passes of the V-cycle.  Chosen per grid by msg123_b200/autotune.py. */
MSG_API int msg_gpu_set_tuning(msg_ctx_t *ctx, int32_t blk_cell, int32_t blk_smooth);

/* Batched ensemble (no counterpart in the reference): advance n independent contexts by
 * nsteps accepted steps each.  nworkers host threads take members from a shared queue
 * and drive each on its own CUDA stream, so members of uneven size and uneven Newton
 * counts run concurrently on the GPU.  rech_until / rech_after: per member (NULL: no
 * schedule).  stats: n entries, may be NULL. */
MSG_API int msg_gpu_ensemble_advance(msg_ctx_t **ctx, int32_t n, int32_t nsteps, const double *rech_until,
                                     const double *rech_after, int32_t nworkers, msg_run_stats_t *stats);

/* Enable (1) or disable (0) the per-phase CUDA-event timers (adds syncs). */
MSG_API int msg_gpu_set_timing(msg_ctx_t *ctx, int32_t on);

#ifdef __cplusplus
}
#endif
#endif /* MSG123_GPU_H */
