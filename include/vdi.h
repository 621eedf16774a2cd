/* vdi.h — C ABI of the B200 implementation of vdropimpact's per-timestep
 * fluid solve.
 *
 * Every entry point returns an int status (VDI_OK = 0). Nothing here exits
 * the process: where the reference calls fatal_error() (common.cc:44-47) the
 * library returns an error status instead.
 *
 * Pointers named d_* are device pointers (CUDA global memory on the current
 * device); pointers named h_* are host pointers. A stream argument of NULL
 * means the legacy default stream. No torch or CUDA C++ types appear here.
 *
 * Array layouts follow the reference:
 *   - a liquid-grid field with ghost layers is (n+4) rows of (m+4) doubles,
 *     row-major, cell (i,j) at [(j+2)*(m+4) + i+2] (fluid_2d.cc:15-18);
 *   - a multigrid solution/source over an m x n grid is m*n values with
 *     ij = i + m*j (mgs_common.cc:8-10);
 *   - tridiagonal systems are four arrays a (sub, a[0] unused), b (diagonal),
 *     c (super, c[n-1] unused) and d (right-hand side, overwritten with the
 *     solution), as tri_solve (tri_solve.hh:6-22).
 */
#ifndef VDI_H
#define VDI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VDI_ABI_VERSION 2

/* ---------------------------------------------------------------- status */
enum vdi_status {
    VDI_OK = 0,
    VDI_ERR_INVALID_ARGUMENT = 1,   /* bad pointer, size or option */
    VDI_ERR_UNSUPPORTED_SIZE = 2,   /* grid the multigrid hierarchy cannot coarsen */
    VDI_ERR_CUDA = 3,               /* a CUDA runtime call failed */
    VDI_ERR_OUT_OF_MEMORY = 4,
    VDI_ERR_MG_NOT_CONVERGED = 5,   /* V-cycle cap reached (mgs_mac.hh:68-70) */
    VDI_ERR_NEWTON_NOT_CONVERGED = 6, /* > 256 Newton steps (gas_layer_solve.cc:204) */
    VDI_ERR_TRI_SINGULAR = 7,       /* zero pivot (dgtsv info != 0, tri_solve.cc:29-32) */
    VDI_ERR_NONFINITE = 8,          /* NaN/Inf in a residual */
    VDI_ERR_CONFIG = 9,             /* configuration text not understood (fileinfo.cc) */
    VDI_ERR_NOT_READY = 10          /* call order violated */
};

/* Returns a static string for a status code. */
const char* vdi_status_string(int status);
/* Returns VDI_ABI_VERSION. */
int vdi_abi_version(void);
/* Detail of the most recent error on the calling thread (static buffer). */
const char* vdi_last_error(void);

/* ------------------------------------------------------------ parameters
 * The drop-impact parameters after fileinfo's unit conversion
 * (fileinfo.cc:142-152), plus the numerical options of this library. */
typedef struct vdi_params {
    int m, n;                 /* liquid grid cells (fileinfo.hh:20-22) */
    int x_sym;                /* symmetric about x=0 (fileinfo.hh:39) */
    int implicit_visc;        /* Crank-Nicolson viscosity (fileinfo.hh:36) */
    double ax, ay, bx, by;    /* domain */
    double mu, rho;           /* liquid dynamic viscosity, density */
    double tmult;             /* timestep padding factor */
    double t_end;             /* simulation duration */
    int nframes;              /* output frames (timestep fitting only) */
    /* gas layer (gas_layer_solve.hh:21-41) */
    double alpha, mug, Pamb, h0, R, V, sigma;
    /* numerical options */
    double mg_rtol;           /* relative residual ||b-Az||/||b|| ending a solve (1e-10) */
    int mg_max_vcycles;       /* V-cycle cap per solve (default 200) */
    int mg_precision;         /* VDI_MG_FP64 or VDI_MG_MIXED */
    int mg_guess;             /* VDI_GUESS_EXTRAPOLATE or VDI_GUESS_LEARNED */
    /* tracers and the non-inertial frame (fileinfo.cc:59, 96-101, 179-191) */
    int ntrace;               /* tracers advected with the flow (0: none) */
    int nif_mode;             /* 0 off; 1 frame velocity at the centre
                                 (nif_center); 2 averaged over columns
                                 [nif_a, nif_b) (nif_range) */
    int nif_a, nif_b;         /* the nif_range window (fileinfo.cc:182-187) */
} vdi_params;

enum vdi_mg_precision {
    VDI_MG_FP64 = 0,          /* FP64 V-cycles */
    VDI_MG_MIXED = 1,         /* FP32 V-cycles inside FP64 iterative refinement */
    VDI_MG_HYBRID = 2         /* FP64 finest level (smoothing, residual, stop test)
                                 with FP32 coarse-grid corrections */
};
enum vdi_mg_guess {
    VDI_GUESS_EXTRAPOLATE = 0, /* linear time extrapolation (mgs_common.cc:17-50) */
    VDI_GUESS_LEARNED = 1,     /* U-Net prediction added to the extrapolation */
    VDI_GUESS_QUADRATIC = 2    /* quadratic extrapolation in time from the last
                                  three solutions (starting iterate only) */
};

/* Parses a vdropimpact .cfg text (fileinfo.cc:11-193; gas_layer_model only)
 * into *out with the default numerical options. */
int vdi_params_from_cfg(const char* cfg_text, vdi_params* out);

/* Run and output options of a .cfg text (fileinfo.cc:56-122): the output
 * flags (fflags bits of the 'output' keyword), restart frequency, tracer count
 * and machine-readable timing flag. The data-driven gas layer
 * (gas_layer_data) is outside the GPU path and returns VDI_ERR_CONFIG. */
typedef struct vdi_run_options {
    unsigned int fflags;      /* 1 u, 2 v, 4 p, 8 pb, 16 pbfull, 32 w, 64 h, 128 fbd,
                                 256 pg, 512 hfull, 1024 fbdfull, 2048 pgfull */
    int restart_freq;         /* frames between restart files (0: none) */
    int ntrace;               /* tracers (fileinfo.hh:26) */
    int mr_time_output;       /* machine-readable timing lines */
} vdi_run_options;
int vdi_run_options_from_cfg(const char* cfg_text, vdi_run_options* out);

/* --------------------------------------------------------- simulation */
typedef struct vdi_sim vdi_sim;

/* fluid_2d::fluid_2d (fluid_2d.cc:14-24): allocates the device state and
 * sets up the four multigrid hierarchies on the current device. */
int vdi_sim_create(const vdi_params* prm, void* stream, vdi_sim** out);
int vdi_sim_destroy(vdi_sim* sim);
/* fluid_2d::init_fields (fluid_2d_sio.cc:14-35) with the gas layer's
 * init_fields (gas_layer_solve.cc:32-53). */
int vdi_sim_init_fields(vdi_sim* sim);
/* fluid_2d::timestep_select (fluid_2d.hh:82-86); also the frame timestep of
 * fluid_2d::solve when interval = t_end/nframes. */
int vdi_sim_timestep_select(const vdi_sim* sim, double interval, double* adt, int* nsteps);
/* fluid_2d::step_forward (fluid_2d.cc:93-405), nsteps times with step dt.
 * Asynchronous with respect to the host unless an error must be reported;
 * the status of device-side checks is read at the end of the call. */
int vdi_sim_step_forward(vdi_sim* sim, double dt, int nsteps);
/* Captures one step_forward(dt) as a CUDA graph with device-side loops for
 * the V-cycles and Newton steps; later vdi_sim_step_forward calls with the
 * same dt replay it. enable=0 returns to eager launches. */
int vdi_sim_use_graph(vdi_sim* sim, int enable);
/* Blocks until queued work finishes; returns the first device-side error. */
int vdi_sim_synchronize(vdi_sim* sim);

/* Host copy of the state the reference writes to a restart file
 * (fluid_2d_sio.cc:97-119, gas_layer_solve.cc:313-331): u, v, p over the
 * ghosted grid ((n+4)*(m+4) each), the gas layer's liquid pressure gp[m+1],
 * shear stress tau[m+4], height h[m], boundary flux fbd[m], gas pressure
 * pg[m+1], height rate ht[m], plus time and Vframe. */
typedef struct vdi_state {
    double time, Vframe;
    double *u, *v, *p;
    double *gp, *tau, *h, *fbd, *pg, *ht;
} vdi_state;
int vdi_sim_get_state(vdi_sim* sim, vdi_state* h_state);
int vdi_sim_set_state(vdi_sim* sim, const vdi_state* h_state);
/* The tracer positions x0, y0, x1, y1, ... (count = 2 * ntrace doubles; the
 * reference's tm array, fluid_2d.hh:49-50). vdi_sim_init_fields places them
 * with the C library's rand() as fluid_2d::init_tracers does
 * (fluid_2d.cc:495-502), so a process that has not called rand() before
 * gets the reference's positions; each step moves them first
 * (fluid_2d::update_tracers, fluid_2d.cc:507-526). */
int vdi_sim_get_tracers(vdi_sim* sim, double* h_xy, long count);
int vdi_sim_set_tracers(vdi_sim* sim, const double* h_xy, long count);

/* The simulation's parameters as they stand (vdi_sim_set_nif_mode changes
 * the frame fields). */
int vdi_sim_get_params(const vdi_sim* sim, vdi_params* out);
/* fluid_2d::init_tracers (fluid_2d.cc:495-502) alone: places the tracers
 * again with the process's rand(), as vdi_sim_init_fields does. */
int vdi_sim_init_tracers(vdi_sim* sim);
/* fluid_2d::update_tracers (fluid_2d.cc:507-526) alone: moves the tracers
 * by dt with the bilinearly interpolated velocity of the current state. */
int vdi_sim_update_tracers(vdi_sim* sim, double dt);
/* fluid_2d::set_nif_mode(mode, w) (declared at fluid_2d.hh:75; the
 * reference gives it no body): switches the non-inertial frame between off
 * (0), the velocity at the centre (1, nif_center, fileinfo.cc:96-98) and the
 * velocity averaged over the columns within w of the axis (2, nif_range w,
 * fileinfo.cc:99-101, 179-191). A window without a column returns
 * VDI_ERR_CONFIG ("Velocity window for non-inertial frame is too small").
 * The next step is captured again. */
int vdi_sim_set_nif_mode(vdi_sim* sim, int mode, double w);

/* gas_layer::update(t, dt) (gas_layer.cc:38-48, with gas_layer_solve's
 * calc_p_and_tau, gas_layer_solve.cc:188-249) alone, on the simulation's
 * current liquid velocity: keeps the previous pressure and shear stress,
 * advances the height, solves the gas pressure by Newton iteration and sets
 * the liquid pressure and the shear stress with its boundary conditions.
 * The simulation clock does not move (fluid_2d::step_forward moves it).
 * Returns VDI_ERR_NEWTON_NOT_CONVERGED or VDI_ERR_TRI_SINGULAR where the
 * reference calls fatal_error. */
int vdi_gas_update(vdi_sim* sim, double dt);
/* gas_layer_solve::init_fields (gas_layer_solve.cc:32-53) alone: the
 * parabolic height, its time derivative -V, zero gas pressure and shear
 * stress. */
int vdi_gas_init_fields(vdi_sim* sim);

/* Per-solver statistics since the last reset (the reference's
 * tgmg_predict::avg_iters and wall-clock counters, mgs_common.hh:47-55). */
typedef struct vdi_stats {
    long steps;
    long solves[4];           /* MAC, FEM, VX, VY */
    long vcycles[4];
    long newton_steps;
    long tri_pivot_fallbacks; /* tridiagonal solves that needed pivoting */
    long height_fixed_point_iters;
    double last_rel_res[4];
    long kernel_launches;     /* kernels this library launched for the counted steps */
} vdi_stats;
int vdi_sim_stats(vdi_sim* sim, vdi_stats* out, int reset);

/* Device pointers to the state arrays (read-only use by callers that keep
 * data on the device). which: 0 u, 1 v, 2 p, 3 gas h, 4 gas pg, 5 gas gp,
 * 6 the last MAC source, 7 the last MAC solution (m*n each), 8 the last FEM
 * source ((m+1)*(n+1)), the contents of fluid_2d::src after a step; the gas
 * layer's 9 previous liquid pressure p_old (m+1), 10 shear stress tau and
 * 11 its previous value tau_old (m+4 each, two ghosts per side), 12 ht and
 * 13 fbd (m each). */
int vdi_sim_device_field(vdi_sim* sim, int which, double** d_ptr, size_t* count);

/* Measurement helper (no reference counterpart): the canonical algorithmic
 * bytes of one solve-loop iteration of each of the simulation's multigrid
 * systems (MAC, FEM, VX, VY; 0 for a system the simulation does not have),
 * with the hierarchies as they stand, for the given vdi_mg_precision. A
 * V-cycle moves (3 (nu1 + nu2) + 4.5) words per point of every level:
 * 8-byte words in FP64, 4-byte words on FP32 levels (every level in
 * VDI_MG_MIXED, the coarse levels in VDI_MG_HYBRID). VDI_MG_MIXED adds its
 * FP64 refinement, 40 bytes per finest point (residual: z, b in, FP32 r
 * out; update: z in and out, FP32 correction in). */
int vdi_sim_vcycle_bytes(const vdi_sim* sim, int precision, double* out4);

/* ----------------------------------------------------------- autotuning
 * Picks, by timing on this GPU with the simulation's own arrays, the launch
 * shape of the per-cell stencil kernels and, for each multigrid system, the
 * level below which the single-CTA coarse cycle replaces the per-level tile
 * kernels. Results are cached in the process per grid (m, n, x_sym,
 * implicit_visc), so simulations of one grid tune once. Restarts the step
 * graph. No reference counterpart (the reference has no tunable kernels). */
typedef struct vdi_tune {
    int blk_x, blk_y;         /* launch shape of the per-cell kernels */
    long cta_limit[4];        /* per system (MAC, FEM, VX, VY): bytes below which
                                 levels run in one CTA; 0 when absent */
    int tiled_levels[4];      /* the resulting per-launch levels (-1: general hierarchy) */
    float stencil_ms;         /* the four advection stages with the chosen shape */
    float vcycle_ms[4];       /* one FP64 V-cycle per system with the chosen cut */
    int from_cache;           /* 1 when an earlier tuning of the same grid was reused */
} vdi_tune;
int vdi_sim_autotune(vdi_sim* sim, vdi_tune* out);
/* Measurement helper (no reference counterpart): mean duration over iters
 * back-to-back launches, with CUDA events on the simulation's stream, of one
 * part of the step: which = 0 the fused advection kernel, 1 the four
 * advection stage kernels, 2 the gas-layer update, 3 the lift-off analysis.
 * The launches use the frame timestep and overwrite the step's intermediate
 * arrays; which = 2 and 3 also advance the gas layer and the lift-off search,
 * so the simulation should be re-initialised (or its state restored) after
 * measuring. */
int vdi_sim_profile(vdi_sim* sim, int which, int iters, float* ms);
/* Applies a tuning (for example one saved from an earlier process). */
int vdi_sim_set_tuning(vdi_sim* sim, const vdi_tune* tune);

/* ---------------------------------------------------------------- batch
 * Independent simulations (a viscosity or impact-velocity sweep over uneven
 * grids) stepped together: one timestep of the batch is one CUDA graph with a
 * branch per simulation, launched once. Each simulation keeps its own arrays
 * and is reachable through vdi_batch_sim for state, statistics and lift-off. No reference
 * counterpart (the reference runs one configuration per process). */
typedef struct vdi_batch vdi_batch;
int vdi_batch_create(const vdi_params* prms, int count, vdi_batch** out);
int vdi_batch_destroy(vdi_batch* batch);
int vdi_batch_size(const vdi_batch* batch);
int vdi_batch_sim(vdi_batch* batch, int k, vdi_sim** out);
int vdi_batch_init_fields(vdi_batch* batch);
/* Autotunes every simulation (grids tune once); out may be NULL or hold
 * count entries. */
int vdi_batch_autotune(vdi_batch* batch, vdi_tune* out);
/* nsteps timesteps of every simulation, simulation k with step dts[k]. The
 * first call with a new set of steps captures the graph. Returns the first
 * simulation's error, naming its index. */
int vdi_batch_step_forward(vdi_batch* batch, const double* dts, int nsteps);

/* ------------------------------------------------------ lift-off search
 * The reference's analysis tool (tt_analysis.cc:97-171) run on the device
 * after every step: the minimum of the gas-layer height profile (as the
 * float32 values a frame file holds, gas_layer_solve.cc:258-282), Gaussian
 * smoothed and interpolated by cubic Hermite pieces (the tool's default) or
 * raw (its -r flag), and the search for the global minimum height, closed
 * once a later minimum exceeds it by 0.5%. The initial state is state 0;
 * state k follows step k*every. On by default (smoothed, every step, no
 * history); init_fields and set_state restart it. */
enum vdi_liftoff_mode {
    VDI_LIFTOFF_OFF = 0,
    VDI_LIFTOFF_SMOOTHED = 1,
    VDI_LIFTOFF_RAW = 2
};
/* Sets the mode, the number of steps between analysed states (every = the
 * frame's step count analyses frames) and the number of states whose
 * (x, height) minimum is kept on the device; restarts the search. */
int vdi_sim_liftoff_setup(vdi_sim* sim, int mode, int every, long history);
typedef struct vdi_liftoff {
    long states;              /* states analysed */
    long min_state;           /* the state of the global minimum (lift-off), -1 before any */
    double min_height, min_x; /* that minimum and its position */
    double interval;          /* time between analysed states (dt * every) */
    double t_rel;             /* min_state * interval - h0 / V (tt_analysis.cc:169-171) */
    double t_rel_ev;          /* min_state * interval - evanescent-field origin */
    double percent;           /* 100 * min_state / (states - 1) */
    int searching;            /* 1 while no later minimum exceeded the global one by 0.5% */
    int ev_found;             /* 1 once a minimum fell below 500 nm (tt_analysis.cc:155-158) */
    double last_x, last_height; /* the last analysed state's minimum */
} vdi_liftoff;
/* Reads the search; h_xmin/h_fmin (may be NULL when cap = 0) receive the
 * first min(cap, states, history) per-state minima. */
int vdi_sim_liftoff(vdi_sim* sim, vdi_liftoff* out, double* h_xmin, double* h_fmin, long cap);
/* The per-profile part alone: the minimum (position, height) of one height
 * profile d_h[m] on cells x_i = ax + (i+1/2) dx (tt_analysis.cc:111-146). */
int vdi_profile_min(int m, double ax, double dx, int mode, const double* d_h, void* stream, double* h_xmin,
                    double* h_fmin);

/* --------------------------------------------------------- multigrid
 * A standalone linear system with the TGMG-style interface the reference's
 * problem classes use (mgs_mac.hh, mgs_fem.hh, visco_impl.hh). */
enum vdi_mg_kind {
    VDI_MG_MAC = 0,           /* mgs_mac.hh:25-50: m x n cells, 5-point */
    VDI_MG_FEM = 1,           /* mgs_fem.hh:42-57: m x n nodes, 9-point FE */
    VDI_MG_VISC_U = 2,        /* visco_impl.hh:28-53, horizontal_vel = true */
    VDI_MG_VISC_V = 3,        /* visco_impl.hh:28-53, horizontal_vel = false */
    VDI_MG_MAC_NEUMANN = 4    /* the MAC operator with a Neumann bottom as well: a pure
                                 Neumann Poisson problem (no reference counterpart; the
                                 reference's systems are all nonsingular). The solve
                                 projects b onto zero mean (its compatibility condition),
                                 stops on the projected residual and returns the
                                 zero-mean solution. */
};
typedef struct vdi_mg vdi_mg;
/* MAC (and MAC_NEUMANN): c1 = dx, c2 = dy (mgs_mac.cc:23-27). FEM: c1 = dx, c2 = dy
 * (mgs_fem.cc:26-30). VISC: c1 = vfx, c2 = vfy, x_sym as visco_impl. */
int vdi_mg_create(int kind, int m, int n, double c1, double c2, int x_sym, void* stream, vdi_mg** out);
int vdi_mg_destroy(vdi_mg* mg);
/* tgmg::setup: builds the level hierarchy (also done by create). */
int vdi_mg_setup(vdi_mg* mg);
/* tgmg::solve_v_cycle: V-cycles on z (initial guess in, solution out) until
 * ||b-Az||_2 <= rtol*||b||_2; precision is a vdi_mg_precision. */
typedef struct vdi_mg_result {
    int vcycles;
    double rel_res;
} vdi_mg_result;
int vdi_mg_solve(vdi_mg* mg, const double* d_b, double* d_z, double rtol, int max_vcycles,
                 int precision, vdi_mg_result* res);
/* tgmg::v_cycle: one FP64 V-cycle on z. */
int vdi_mg_v_cycle(vdi_mg* mg, const double* d_b, double* d_z);
/* r = b - A z (the residual tgmg::output_res writes) and its 2-norm. */
int vdi_mg_residual(vdi_mg* mg, const double* d_b, const double* d_z, double* d_r, double* norm);
/* y = A z, the operator of the problem class (a_cc*z + mul_a). */
int vdi_mg_apply(vdi_mg* mg, const double* d_z, double* d_y);
/* Measurement helper: launches, iters times on d_b, d_z between two CUDA
 * events on the system's stream, which = 0 the finest-level
 * pre-smoothing/restriction kernel, 1 the finest prolongation/post-smoothing
 * kernel, 2 a whole FP64 V-cycle (the ms per V-cycle that mg_test.cc:36-43
 * reports), 3 the single-launch coarse cycle alone; in the mixed precision's
 * refinement, 4 the finest FP32 pre-smoothing kernel (from zero), 5 the
 * finest FP32 post-smoothing kernel, 6 the FP64 residual pass that writes
 * the FP32 source; returns the mean duration and the algorithmic bytes per
 * launch (0 for which = 3). */
int vdi_mg_profile(vdi_mg* mg, int which, int iters, const double* d_b, double* d_z, float* ms_per_launch,
                   double* bytes_per_launch);
/* The coarse levels of a V-cycle (of the given vdi_mg_precision) that run in
 * one launch: the first such level (level 0 the finest; -1 when the
 * hierarchy has none) and the CTAs of that launch (1: a single CTA; 8 or
 * 16: a thread-block cluster whose CTAs hold row slabs of every level; 0:
 * that level is solved exactly by a dense inverse applied over the whole
 * GPU, as FEM hierarchies do when it has at most 3072 unknowns; -1: that
 * level is solved exactly by cosine transforms in x and one tridiagonal
 * system per mode in y, as separable MAC and FEM hierarchies do at their
 * first level of at most 40000 unknowns). No reference counterpart. */
int vdi_mg_coarse_cycle(const vdi_mg* mg, int precision, int* first_level, int* ctas);
/* Which kernel runs the tiled levels, read once per process from
 * VDI_MG_TILE: 0 the shared-memory tiles (default), 1 register-blocked
 * tiles at two CTAs per SM ("reg"), 2 the same at one CTA per SM ("reg1"),
 * 3 the persistent TMA-fed register tile on FP64 cell-centred levels, the
 * others as in 0 ("tma"). *persistent_launches (if not null) receives the
 * persistent tile's launches issued so far, a captured graph's once. */
int vdi_mg_tile_path(long long* persistent_launches);

/* ------------------------------------------------------------ U-Net
 * The learned initial guess has no counterpart in the reference. A small
 * convolutional U-Net maps the RMS-normalised residual of the extrapolated
 * guess, on a coarsened H x W grid (H a multiple of 8, W of 16), to a
 * normalised correction. Inputs and outputs are FP32 device arrays of batch
 * x H x W values; parameters are BF16 on the device with FP32 master copies. */
typedef struct vdi_unet vdi_unet;
int vdi_unet_create(int H, int W, int batch, unsigned seed, void* stream, vdi_unet** out);
int vdi_unet_destroy(vdi_unet* net);
long vdi_unet_param_count(const vdi_unet* net);
int vdi_unet_forward(vdi_unet* net, const float* d_in, float* d_out, int batch);
/* Which tensor-core path the forward and input-gradient convolutions take:
 * 1 tcgen05.mma with TMEM accumulators (the default), 0 mma.sync
 * (VDI_UNET_TC=0, read once per process). */
int vdi_unet_tensor_path(void);
/* One Adam step on the mean squared error of the output against d_target. */
int vdi_unet_train_step(vdi_unet* net, const float* d_in, const float* d_target, int batch, float lr, float* h_loss);
/* Loss and the weight gradient of one layer ([9][cout][cin], FP32) without
 * updating the parameters (gradient checks). */
int vdi_unet_gradients(vdi_unet* net, const float* d_in, const float* d_target, int batch, int layer, float* h_grad,
                       float* h_loss);
/* All parameters (per layer: weights [9][cout][cin], then biases), FP32, to
 * (to_device = 1) or from the device. */
int vdi_unet_params(vdi_unet* net, float* h_buf, long count, int to_device);
/* Attaches a trained network to the MAC solve of a simulation as its
 * VDI_GUESS_LEARNED initial guess: the network runs on the residual of the
 * extrapolated guess restricted by factor (2 or 4), and its output times
 * out_scale * rms(residual) / xxsp, prolonged back, is added to the guess. */
int vdi_sim_attach_unet(vdi_sim* sim, vdi_unet* net, int factor, double out_scale);

/* The learned guess for a standalone MAC solve (no reference counterpart):
 * with r = b - A z for the current z, adds to z the network's prediction of
 * A^-1 r: r restricted by factor and divided by its RMS is the input, and
 * the output times scale * rms(r), prolonged back, is the correction (scale
 * is the network's output scale over xxsp). Then solve from z as usual. */
int vdi_unet_guess(vdi_unet* net, vdi_mg* mg, int factor, double scale, const double* d_b, double* d_z);

/* vdi_mg_solve_noalloc has no counterpart in the reference. It is an FP64
 * multigrid solve of the systems of vdi_mg_create + vdi_mg_solve for callers
 * that must not allocate device memory, such as an application that owns
 * every device allocation itself or code running where an allocation would
 * stall or fail. It allocates nothing: besides the caller's d_b and d_z it
 * uses one static device array of about 5 MB that every GPU loading the
 * library holds until exit. Grids are limited to 262144 unknowns (m*n);
 * larger ones return VDI_ERR_UNSUPPORTED_SIZE. Its coarsest level is
 * smoothed rather than solved with a precomputed inverse, so its V-cycle
 * count can exceed vdi_mg_solve's (about twice on a 641 x 385 FEM grid,
 * 17 against 9); it stops on the same residual test.
 * The first call on a device looks up the array's device address and should
 * come before any stream capture. Calls share the array: two calls that
 * overlapped on the GPU would race on it. The entry point holds a
 * process-wide lock for the whole call and returns only once its solve has
 * finished, so calls from different host threads run one after another.
 * Arguments are those of vdi_mg_create and vdi_mg_solve; stream may be
 * NULL. */
int vdi_mg_solve_noalloc(int kind, int m, int n, double c1, double c2, int x_sym, const double* d_b, double* d_z,
                         double rtol, int max_vcycles, void* stream, vdi_mg_result* res);

/* ------------------------------------------------------- tridiagonal
 * tri_solve::solve_lapack (tri_solve.cc:24-33): solves the n x n system in
 * place (solution in d_d) on the GPU by cyclic reduction, falling back to
 * Gaussian elimination with partial pivoting when a row is not diagonally
 * dominant. a, b, c are overwritten. *pivoted is set to 1 when the fallback
 * ran (may be NULL). */
int vdi_tri_solve(int n, double* d_a, double* d_b, double* d_c, double* d_d, void* stream, int* pivoted);

#ifdef __cplusplus
}
#endif

#endif
