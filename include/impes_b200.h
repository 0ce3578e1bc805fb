/*
 * impes_b200.h -- C ABI of the B200-native IMPES pressure/saturation path.
 *
 * The library replaces the hot path of researchim-ai/oil-simulator-py's IMPES
 * time step: pressure assembly, the Ruge-Stueben AMG pressure solve and the
 * explicit three-phase saturation update.  Every entry point takes plain device
 * pointers and sizes (caller-owned I/O buffers, float64 unless noted), returns
 * an int status (IMPES_OK = 0) and enqueues its work on the given CUDA stream
 * (`stream` is a cudaStream_t passed as void*; NULL = legacy default stream).
 * On failure `impes_last_error()` returns a message (thread-local).
 *
 * Layout: cell fields are flat arrays over c = (i*ny + j)*nz + k (z fastest),
 * the reference's flatten order (src/simulator/simulation.py:804-816).
 * Matrices are CSR with int32 row pointers / columns, sorted columns.
 */
#ifndef IMPES_B200_H
#define IMPES_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum {
  IMPES_OK = 0,
  IMPES_ERR_ARG = 1,           /* invalid argument / size                         */
  IMPES_ERR_CUDA = 2,          /* CUDA runtime error                              */
  IMPES_ERR_NOT_CONVERGED = 3, /* Krylov/V-cycle hit its iteration cap            */
  IMPES_ERR_NAN = 4,           /* NaN/Inf detected in inputs or iterates          */
  IMPES_ERR_BAD_CSR = 5,       /* malformed CSR (row pointers, columns)           */
  IMPES_ERR_COARSENING = 6,    /* no level could be built                         */
  IMPES_ERR_OOM = 7,           /* device allocation failed                        */
  IMPES_ERR_TIMEOUT = 8,       /* a bounded device wait expired                   */
  IMPES_ERR_SINGULAR = 9,      /* coarsest LU broke down                          */
  IMPES_ERR_STATE = 10         /* call out of order (e.g. update before setup)    */
};

const char* impes_last_error(void);
int impes_abi_version(void);

/* ================================================================== AMG ===
 * Classical Ruge-Stueben AMG with the reference's algorithm
 * (src/solver/classical_amg.py): strength of connection (:34-82), C/F split
 * (:85-146), RS interpolation with F-F distribution, weak correction, row
 * normalisation and energy-minimising blend (:149-427, :1469-1501), Galerkin
 * P^T A P (:519-657), equilibration (:763-788), l1-Jacobi smoothing (:1016-1035),
 * V-cycle with a pinned dense coarsest solve (:1037-1106).
 */
typedef struct impes_amg impes_amg;

typedef struct {
  double theta;                   /* strength threshold, 0.25                    */
  int max_levels;                 /* 10                                          */
  int coarsest_size;              /* 100 (ClassicalAMG) / 200 (amg_solve)        */
  int nullspace_dim;              /* 0..3 (3)                                    */
  double nullspace_blend;         /* 0.6                                         */
  double nullspace_reg;           /* 1e-6                                        */
  double equilibration_threshold; /* 1e-6                                        */
  uint32_t tiebreak_seed;         /* C/F tie-break stream (replaces torch.rand)  */
  int mixed_precision;            /* 1: also keep an fp32 copy for the V-cycle   */
  /* Interpolation truncation (no counterpart in the reference; 0 / 0.0 keep the
   * reference's interpolation): after the energy blend each F row of P keeps at
   * most p_max_elements entries (0 = no cap), drops entries below
   * p_trunc_factor times the row's largest, and is rescaled to its old row sum. */
  int p_max_elements;
  double p_trunc_factor;
  /* Smoother of the V-cycle: IMPES_SMOOTHER_L1_JACOBI (the reference's, 0.7 *
   * l1-Jacobi) or IMPES_SMOOTHER_CHEBYSHEV (no counterpart in the reference):
   * the Chebyshev iteration for diag(l1 weights) A on [cheb_lower * lmax, lmax],
   * lmax its Gershgorin bound, one step per sweep the V-cycle would make. */
  int smoother;
  double cheb_lower;              /* 0.3 when <= 0                               */
  /* Levels of at most light_sweep_rows rows smooth once before and once after
   * their coarse-grid correction instead of the reference's three and two
   * (0: every level as the reference).  On small levels each sweep costs a
   * kernel launch's latency rather than its bytes, so this trades a little
   * smoothing for fewer launches; it changes the preconditioner, not the answer
   * a Krylov solve stops on.  The fused V-cycle tails are off when it is set. */
  int light_sweep_rows;
} impes_amg_params;

enum { IMPES_SMOOTHER_L1_JACOBI = 0, IMPES_SMOOTHER_CHEBYSHEV = 1 };

typedef struct {
  int n;
  int nnz;
  int p_cols;      /* coarse size (0 on the coarsest level) */
  int p_nnz;
  int is_coarsest;
  int col_index_bytes;   /* 2 or 4: column storage of the smoothing/residual passes */
  int col_row_relative;  /* 1: 16-bit columns hold col - row + 32768              */
  int lanes[6];          /* autotuned lanes per row of the kernels on A, R (restriction)
                            and P (prolongation): [0..2] fp64, [3..5] fp32; 0 = rule  */
  int layout[2];         /* storage the sweeps and residuals on A read: 0 CSR, 1 the
                            level's SELL-32 (sliced ELLPACK) copy, 2 its DIA (one array
                            per diagonal) copy, 3 the DIA copy of a grid's 7-point
                            stencil with two sweeps (and the residual) per launch on
                            grid tiles; [0] fp64, [1] fp32                            */
  int fused_tail;        /* 1: the level's fp32 V-cycle runs inside the one-CTA
                            shared-memory tail launch, 2: inside the cluster tail     */
} impes_amg_level_desc;

/* Norms for Krylov stopping tests. */
enum {
  IMPES_NORM_EQUILIBRATED = 0, /* ||D^-1/2 r|| / ||D^-1/2 b|| (classical_amg.py:1136-1145) */
  IMPES_NORM_JACOBI = 1        /* ||D^-1 r||   / ||D^-1 b||, D = |diag A|               */
};

typedef struct {
  double tol;
  int restart;        /* FGMRES restart length                      */
  int max_iters;      /* total iteration cap                        */
  int norm;           /* IMPES_NORM_*                               */
  int precision;      /* 0: fp64 V-cycle, 1: fp32 V-cycle (mixed)   */
  int use_x0;         /* 1: x holds an initial guess; 2 (impes_step only): the
                         pressure extrapolated linearly in time from the last
                         two accepted steps (the current one on the first);
                         3 (impes_step only): quadratically from the last
                         three (linearly while only two are known)            */
} impes_krylov_params;

typedef struct {
  int iterations;     /* preconditioner applications (V-cycles)     */
  int restarts;
  int converged;
  double rel_res;     /* final estimate in the selected norm        */
  double true_rel_res;/* explicitly recomputed in the selected norm */
} impes_krylov_stats;

/* ClassicalAMG.__init__ parameters (classical_amg.py:699-725). */
int impes_amg_create(impes_amg** out, const impes_amg_params* params);
int impes_amg_destroy(impes_amg* h);

/* ClassicalAMG.__init__ (classical_amg.py:699-938): build the hierarchy from a
 * device CSR (n rows, nnz entries, float64 values). */
int impes_amg_setup(impes_amg* h, int n, int nnz, const int* rowptr, const int* col,
                    const double* val, void* stream);

/* ClassicalAMG.update_matrix (classical_amg.py:1308-1392): new values on the
 * same pattern; frozen P, fresh equilibration and Galerkin products. */
int impes_amg_update(impes_amg* h, const double* val, void* stream);

/* ClassicalAMG.solve (classical_amg.py:1108-1155): stand-alone V-cycles from
 * x0 = 0 until ||r_s||/||b_s|| < tol or max_cycles.  b, x: device, length n.
 * cycles/rel_res: host outputs (may be NULL).  norm: IMPES_NORM_EQUILIBRATED (the
 * reference's test) or IMPES_NORM_JACOBI. */
int impes_amg_solve_vcycles(impes_amg* h, const double* b, double* x, double tol,
                            int max_cycles, int* cycles, double* rel_res, int norm, void* stream);

/* The stand-alone V-cycle solve above, for callers that must not allocate
 * device memory during a solve -- for example a host that reserves the GPU's
 * memory up front for its own pool, or one that cannot afford the device-wide
 * synchronisation that cudaFree implies.  (No counterpart in the reference.)
 * impes_amg_solve_vcycles allocates and frees three n-vectors on every call;
 * this variant keeps them in a 6 MiB static device array instead and makes no
 * allocation, so n is limited to 262144 rows (larger n returns IMPES_ERR_ARG).
 * Every GPU that loads the library holds that array until the process exits.
 * Every call on a device shares it: calls that overlap on the GPU (several
 * streams or threads) race, so serialise them.  Nothing in the array needs to
 * start at zero (each call writes before it reads).  The first call on each
 * device (and the first after that device's context was re-created, e.g. by
 * cudaDeviceReset) looks up the array's device address; make that first call
 * before any stream capture.  Results equal impes_amg_solve_vcycles'. */
int impes_amg_solve_vcycles_noalloc(impes_amg* h, const double* b, double* x, double tol,
                                    int max_cycles, int* cycles, double* rel_res, int norm,
                                    void* stream);

/* ClassicalAMG.apply (classical_amg.py:1157-1180): `cycles` V-cycles, then
 * continue up to apply_max_cycles while ||r||/||b|| >= apply_tol. */
int impes_amg_apply(impes_amg* h, const double* b, double* x, int cycles, double apply_tol,
                    int apply_max_cycles, void* stream);

/* One V-cycle on the equilibrated system: x = V(0, b_s) (classical_amg.py:1037). */
int impes_amg_vcycle_scaled(impes_amg* h, const double* b_scaled, double* x_scaled,
                            int precision, void* stream);

/* Flexible GMRES preconditioned by one V-cycle per iteration (no reference
 * counterpart: the reference runs stand-alone V-cycles; its test and docs name
 * "gmres_amg").  Solves A x = b (unscaled); float64 Krylov basis,
 * orthogonalisation, true residual; V-cycle in fp64 or fp32. */
int impes_amg_fgmres(impes_amg* h, const double* b, double* x, const impes_krylov_params* kp,
                     impes_krylov_stats* stats, void* stream);

/* Hierarchy introspection (ClassicalAMG.levels, .Dhalf_inv). */
int impes_amg_num_levels(impes_amg* h, int* nlev);
int impes_amg_level_info(impes_amg* h, int lvl, impes_amg_level_desc* info);
/* Instrumentation (no reference counterpart): mean device time in microseconds
 * of one l1-Jacobi sweep, residual, restriction and prolongation of every level
 * (precision 0: fp64, 1: fp32), each launched `reps` times back to back on the
 * level's work vectors; out_host[4 * level + k], 0 on the coarsest level.
 * Overwrites the hierarchy's work vectors; synchronises the stream. */
int impes_amg_profile_levels(impes_amg* h, int precision, int reps, double* out_host, void* stream);
/* Instrumentation: whole IMPES steps this handle holds as CUDA graphs
 * (impes_step from the second FGMRES step on) and whether a capture was
 * refused, after which its steps stay host-driven. */
int impes_amg_step_graphs(impes_amg* h, int* graphs, int* capture_refused);
/* Copy level `lvl` into caller device buffers (any pointer may be NULL). */
int impes_amg_level_export(impes_amg* h, int lvl, int* A_rowptr, int* A_col, double* A_val,
                           double* inv_relax, int* P_rowptr, int* P_col, double* P_val,
                           void* stream);
/* Equilibration state: *enabled = 1 and dhalf_inv filled (device, n) when on. */
int impes_amg_equilibration(impes_amg* h, double* dhalf_inv, int* enabled, void* stream);

/* ================================================================ IMPES ===
 * Model = Reservoir + Fluid + WellManager + the IMPES parts of Simulator
 * (src/simulator/{reservoir,fluid,well,pvt,simulation}.py).
 */
typedef struct impes_model impes_model;

typedef struct {
  int nx, ny, nz;
  double dx, dy, dz;                       /* m                                    */
  double mu_o, mu_w, mu_g;                 /* Pa*s (fluid.py:31-33), no-PVT case   */
  double rho_o_ref, rho_w_ref, rho_g_ref;  /* kg/m3 (fluid.py:36-38)               */
  double c_o, c_w, c_g, c_r;               /* 1/Pa (fluid.py:41-44)                */
  double cf;                               /* (c_o+c_w+c_g+c_r)/3 (fluid.py:47)    */
  int relperm_model;                       /* 0 Corey, 1 Stone II (fluid.py:62)    */
  double nw, no, ng, now, nog;             /* exponents (fluid.py:63-70)           */
  double ko_end_w, ko_end_g;
  double sw_cr, so_r, sg_cr;
  double pc_scale, pc_exponent;            /* fluid.py:97-105 (Pa)                 */
  double pc_og_scale, pc_og_exponent;      /* fluid.py:108-110                     */
  double gravity;                          /* 9.81 (simulation.py:81)              */
  double global_rate_scale;                /* simulation params                    */
  double max_saturation_change;            /* 0.05                                 */
  int max_substeps;                        /* 20                                   */
  int pvt_rows;                            /* 0 = no PVT table                     */
} impes_model_desc;

enum { IMPES_PHASE_WATER = 0, IMPES_PHASE_GAS = 1 };
enum { IMPES_SURF_OIL = 0, IMPES_SURF_WATER = 1, IMPES_SURF_GAS = 2, IMPES_SURF_LIQUID = 3 };
enum { IMPES_LIM_WOPR = 1, IMPES_LIM_WLPR = 2, IMPES_LIM_WGPR = 4, IMPES_LIM_LIQR = 8 };

/* One well (well.py:10-55, both schemas of WellManager :77-92). */
typedef struct {
  int i, j, k;
  int is_injector;      /* 1 injector, 0 producer                    */
  int control_bhp;      /* 0 rate (m3/day), 1 bhp (MPa)              */
  double value;         /* control_value as in the JSON              */
  double well_index;    /* Peaceman index (well.py:44-51)            */
  int injected_phase;   /* IMPES_PHASE_*                             */
  int surface_rate;     /* rate_type == "surface"                    */
  int surface_phase;    /* IMPES_SURF_* (default liquid)             */
  int limit_mask;       /* IMPES_LIM_* bits                          */
  double limits[4];     /* wopr, wlpr, wgpr, liqr (m3/day)           */
  int has_bhp_min;
  double bhp_min;       /* MPa                                       */
} impes_well_desc;

/* Per-well diagnostics after a step (well.py:53-55). */
typedef struct {
  int last_mode;          /* -1 unset, 0 rate, 1 bhp (pressure step auto-switch) */
  int has_q_total;
  double last_q_total;    /* m3/s                                                */
  int has_surface_rates;
  double surface_rates[4];/* oil, water, gas, liquid (m3/day)                    */
} impes_well_state;

typedef struct {
  int substeps;           /* N of the saturation update                 */
  double mass_balance[6]; /* water in/out, oil in/out, gas in/out (kg)  */
  double component[6];    /* oil in/out/accum, gas in/out/accum (sm3)   */
} impes_sat_stats;

/* Model construction: Simulator.__init__ transmissibilities
 * (simulation.py:52-74) and pore volume (reservoir.py:48-50).  kx, ky, kz (m^2),
 * poro: device arrays of nx*ny*nz.  pvt: host array pvt_rows x 9 columns
 * (P MPa, Bo, Bw, Bg, mu_o cP, mu_w cP, mu_g cP, Rs, Rv) or NULL (pvt.py:18-46). */
int impes_model_create(impes_model** out, const impes_model_desc* desc,
                       const impes_well_desc* wells, int nwells, const double* pvt,
                       const double* kx, const double* ky, const double* kz,
                       const double* poro, void* stream);
int impes_model_destroy(impes_model* m);

/* Static 7-point CSR pattern as coalesce().to_sparse_csr() orders it
 * (simulation.py:1546-1580): rowptr (N+1), col (nnz).  nnz via impes_model_nnz. */
int impes_model_nnz(impes_model* m, int* n, int* nnz);
int impes_csr_pattern(impes_model* m, int* rowptr, int* col, void* stream);
/* Flat cell index of each well, (i*ny + j)*nz + k (simulation.py:1629-1630). */
int impes_well_cells(impes_model* m, int* cells_host);
/* New control values of the wells (rate m3/day or BHP MPa, in well order, host
 * array of nwells), as when a caller assigns Well.control_value between steps
 * (rl_env.py:127-140).  Takes effect from the next assembly. */
int impes_model_set_well_values(impes_model* m, const double* values, int nwells, void* stream);
/* Device transmissibilities (F face values, x then y then z) and pore volume. */
int impes_model_export_static(impes_model* m, double* tx, double* ty, double* tz, double* pv,
                              void* stream);

/* Pressure assembly, _impes_pressure_step steps 1-4 (simulation.py:867-904,
 * 1546-1660): matrix values into the static pattern and the right-hand side. */
int impes_assemble(impes_model* m, const double* p, const double* sw, const double* sg,
                   double dt, double* csr_val, double* rhs, void* stream);

/* Explicit saturation update, _impes_saturation_step (simulation.py:968-1544).
 * p_new: device (N); sw, sg updated in place, so = 1 - sw - sg written.
 * Mass/component balances accumulate inside the model; stats (host, may be
 * NULL) receives the running totals after a stream sync. */
int impes_saturation(impes_model* m, const double* p_new, double* sw, double* sg, double* so,
                     double dt, impes_sat_stats* stats, void* stream);

/* One full IMPES step, _impes_step (simulation.py:822-865): assemble, AMG
 * setup on first use / update_matrix afterwards, pressure solve
 * (solver = 0: stand-alone V-cycles to kp->tol in the equilibrated norm, the
 * reference's "amg" branch; solver = 1: FGMRES per kp; solver = 2: the
 * reference's default Jacobi-PCG from zero to sqrt(r.M^-1 r) < kp->tol within
 * kp->max_iters, then once more with 10x the tolerance and 4x the iterations,
 * simulation.py:931-966 -- amg may be NULL), then the saturation update.  p is
 * replaced by the new pressure; on a missed tolerance p is restored and
 * IMPES_ERR_NOT_CONVERGED returned.  kstats/sstats may be NULL. */
int impes_step(impes_model* m, impes_amg* amg, double* p, double* sw, double* sg, double* so,
               double dt, int solver, const impes_krylov_params* kp, int max_cycles,
               impes_krylov_stats* kstats, impes_sat_stats* sstats, void* stream);

/* Simulator._solve_pressure_cg_pytorch (simulation.py:1662-1697): Jacobi-
 * preconditioned CG on a CSR matrix (device arrays, n rows) from x = 0, stopping
 * when sqrt(r . D^-1 r) < tol (absolute) or after max_iter iterations.  x is
 * written; iterations, converged and the last r . D^-1 r (rz) may be NULL. */
int impes_pcg_solve(int n, const int* rowptr, const int* col, const double* val, const double* b,
                    double* x, double tol, int max_iter, int* iterations, int* converged,
                    double* rz, void* stream);

/* Running balances and per-well diagnostics (host outputs; syncs the stream). */
int impes_model_balances(impes_model* m, impes_sat_stats* stats, void* stream);
int impes_model_reset_balances(impes_model* m, void* stream);
int impes_well_states(impes_model* m, impes_well_state* out_host, void* stream);

/* ======================================================== instrumentation ===
 * CUDA-event timers around the phases of the step (no reference counterpart:
 * the reference prints perf_counter timings, classical_amg.py:799-875).  Events
 * are recorded on the stream of the timed call; collecting synchronises.
 * Not thread-safe: one timing session per process. */
enum {
  IMPES_PH_ASSEMBLE = 0,   /* K1 pressure assembly                        */
  IMPES_PH_SATURATION = 1, /* K4 saturation update (wells + flux + substeps) */
  IMPES_PH_GALERKIN = 2,   /* update_matrix: equilibration + P^T A P, all levels */
  IMPES_PH_VCYCLE = 3,     /* one V-cycle from level 0                    */
  IMPES_PH_SMOOTH_L0 = 4,  /* one l1-Jacobi sweep on level 0              */
  IMPES_PH_SPMV_L0 = 5,    /* FGMRES operator product on level 0          */
  IMPES_PH_ORTHO = 6,      /* FGMRES Gram-Schmidt of one iteration        */
  IMPES_PH_SOLVE = 7,      /* whole pressure solve                        */
  IMPES_PH_SMOOTH_WIDE = 8,/* one l1-Jacobi sweep on a level with > 96 nnz per row (warps per row) */
  IMPES_PH_TILE_L0 = 9,    /* two l1-Jacobi sweeps (and the residual) on level 0's grid tiles, one launch */
  IMPES_NUM_PHASES = 10
};
typedef struct {
  long long count[10];  /* timed launches per phase                     */
  double ms[10];        /* summed device time per phase                 */
  double bytes[10];     /* summed algorithmic bytes per phase           */
} impes_timing;
int impes_timing_enable(int on);
int impes_timing_collect(impes_timing* out);
/* Kernel launches issued by the library since load. */
unsigned long long impes_kernel_launches(void);

/* ----------------------------------------------------------------- ensemble
 * Independent realisations stepped concurrently (no counterpart in the
 * reference, whose callers loop over Simulator.run_step).  Member m has its own
 * model and AMG handle and its own state arrays; each member's numerics are
 * those of impes_step on that member alone (FGMRES solver with *kp).  A pool of
 * `workers` host threads, each with its own CUDA stream on the calling thread's
 * device, takes members largest first (cells[m]) and runs all `steps` steps of
 * dt seconds.  Returns IMPES_OK, or the status of the first failing member
 * (impes_last_error names it); per-member results are in stats[members].
 * span_ms (may be NULL) receives the device time from before the first
 * member's first kernel to after the last member's last kernel.
 * Handles of different members must be distinct. */
typedef struct {
  int status;            /* IMPES_OK or this member's error                 */
  int steps_done;
  long long iterations;  /* FGMRES iterations over its steps                */
  double device_ms;      /* device time of its steps on its worker's stream */
  int worker;            /* host thread that ran it                         */
} impes_ensemble_member_stats;
int impes_ensemble_run(impes_model** models, impes_amg** amgs, double** p, double** sw,
                       double** sg, double** so, const int* cells, int members, int steps,
                       double dt, const impes_krylov_params* kp, int workers,
                       impes_ensemble_member_stats* stats, double* span_ms);

/* ------------------------------------------------------------------ adjoint
 * Discrete adjoint of the IMPES step (no counterpart in the reference).
 * Objective J = sum over steps and producers of (q_o - q_target)^2, q_o the
 * producer oil rate (m3/day) from the flux balance of its pressure row,
 *   q = sum_f c_f (p_nb - p_c) - PV ct/dt (p_c - p_prev) + Qg_c,
 * times the oil fractional flow at the step's starting saturation.  This is
 * the well's WI*lambda_t*(p - p_bhp) (simulation.py:1297) written without its
 * round-off.  Gradients are with respect to ln k (kx, ky, kz of a cell scaled
 * together) and porosity.  Scope: oil-water (s_g = 0) without PVT tables or
 * capillarity, Corey relative permeability, no bhp_min switching; other models
 * return IMPES_ERR_ARG.  The runs step internal copies of the state (the
 * caller's p, sw are not touched by impes_adjoint_gradient) and use the model's
 * and the AMG handle's work space: the model's mass balances are restored, the
 * hierarchy is left holding the values of some step's matrix. */
typedef struct {
  double J;                       /* objective of the forward run                 */
  long long forward_iterations;   /* FGMRES iterations, forward run + recomputation */
  long long adjoint_iterations;   /* FGMRES iterations of the adjoint solves       */
  double forward_ms;              /* device time of the forward run                */
  double reverse_ms;              /* device time of the reverse sweep (recomputation included) */
  int checkpoints;                /* state checkpoints kept                        */
  int recomputed_steps;           /* forward steps recomputed from checkpoints     */
} impes_adjoint_stats;
/* Producers observed by the objective (wells of type producer, in well order). */
int impes_adjoint_num_producers(impes_model* m, int* n);
/* Forward run of `steps` steps from (p, sw) in place (s_g = 0), writing the
 * producer oil rates to rates_host[steps * nprod] (may be NULL). */
int impes_adjoint_rates(impes_model* m, impes_amg* amg, double* p, double* sw, int steps,
                        double dt, const impes_krylov_params* kp, double* rates_host,
                        void* stream);
/* J and dJ/dln k, dJ/dphi (device arrays of N) for the run of `steps` steps
 * from (p0, sw0).  States are checkpointed every `checkpoint_every` steps
 * (0: keep all) and recomputed segment by segment in the reverse sweep; the
 * adjoint pressure solve reuses the forward hierarchy (A is symmetric).
 * kx, ky, kz are the model's permeabilities (m^2, device).  target_host and
 * rates_host (may be NULL) hold steps * nprod rates in m3/day. */
int impes_adjoint_gradient(impes_model* m, impes_amg* amg, const double* p0, const double* sw0,
                           const double* kx, const double* ky, const double* kz, int steps,
                           int checkpoint_every, double dt, const impes_krylov_params* forward,
                           const impes_krylov_params* adjoint, const double* target_host,
                           double* rates_host, double* g_lnk, double* g_poro,
                           impes_adjoint_stats* stats, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* IMPES_B200_H */
