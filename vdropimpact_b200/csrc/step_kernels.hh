// Declarations shared between the step kernels, the gas-layer kernel and
// the simulation driver.
#pragma once

#include "vdi_internal.hh"

namespace vdi {

/** Grid and physical constants of the liquid domain (fluid_2d.hh:23-44). */
struct Grid {
    int m, n;
    int x_sym, implicit_visc;
    int blk_x, blk_y;          // launch shape of the per-cell kernels (autotuned)
    double ax, ay, bx, by, dx, dy, xsp, ysp, xxsp, yysp;
    double rho, rhoinv, mu, muinv, viscfac;
};

/** Device pointers of the per-cell fields, each over the ghosted grid.
 * Edge set 1 (ud..vu) holds stages 1-2 and then the final upwinded values;
 * edge set 2 (ud2..vu2) holds the stage-4 extrapolations. */
struct Fields {
    double *u, *v, *p;
    double *ux, *uy, *vx, *vy;
    double *ud, *vd, *ul, *vl, *ur, *vr, *uu, *vu;
    double *ud2, *vd2, *ul2, *vl2, *ur2, *vr2, *uu2, *vu2;
    double *fc0, *fc1;
};

/** Gas-layer arrays (gas_layer.hh:31-39, gas_layer_solve.hh:51-65). */
struct Gas {
    double *gp, *gp_old, *tau, *tau_old;
    double *h, *hx, *ht, *fbd, *pg, *pg_old;
};

/** Gas-layer parameters (gl_params, gas_layer_solve.hh:21-41). */
struct GasPrm {
    int m, x_sym;
    double ax, dx, xsp, xxsp;
    double alpha, mu, Pamb, R, sigma;
};

/** Counters written by the gas-layer kernel. */
struct GasStats {
    long long updates;
    long long newton_steps;
    long long pivot_fallbacks;
    long long fixed_point_iters;
    long long sequential_fallbacks;
};

/** Time-extrapolation history of one solver (mgs_common.hh:21-36). */
struct GuessHist {
    int scount;
    unsigned arrive;    // blocks of the current guess launch that have read the history
    double t_prev, t0;
    double t_prev2;     // time of the third-latest solution (quadratic guess)
    int head;           // quadratic guess: 1 when zprev2 holds the t_prev solution
};

/** A read-only view of a cell array with an arbitrary pitch and origin. */
struct CellView {
    const double* p;
    int pitch, off;
    __device__ __forceinline__ double at(int i, int j) const { return p[off + i + pitch * j]; }
};

int launch_stage1(cudaStream_t s, const Grid& g, const Fields& f, double dt);
int launch_stage2(cudaStream_t s, const Grid& g, const Fields& f);
int launch_stage34(cudaStream_t s, const Grid& g, const Fields& f, double dt);
int launch_stage5_src(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs, double dt, double* src);
/** Stages 1-5 of the advection in one kernel (all but the bottom-row gas
 * term of the MAC source), and that term. */
int launch_advect(cudaStream_t s, const Grid& g, const Fields& f, double dt, double* src);
int launch_mac_src_bottom(cudaStream_t s, const Grid& g, const Gas& gs, double dt, double* src);
int launch_mac_advect(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs, const double* q, double dt,
                      double* d_time);
int launch_inviscid_bc(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs, double dt);
int launch_viscous_bc(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs);
int launch_visc_rhs(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs, double vfx, double vfy,
                    double* su, double* sv);
int launch_fem_rhs(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs, CellView c0, CellView c1, double dt,
                   double a_cc_edge, double a_cc_mid, double* src);
int launch_vel_update(cudaStream_t s, const Grid& g, const Fields& f, CellView c0, CellView c1, const double* z,
                      double dt);
/** fluid_2d::update_tracers (fluid_2d.cc:507-526) for ntrace tracers. */
int launch_tracers(cudaStream_t s, const Grid& g, const Fields& f, double* tm, int ntrace, double dt);
/** fluid_2d::adjust_frame (fluid_2d_sio.cc:228-253): mode 1 (nif_center) or
 * 2 (nif_range over columns [a, b)); vacc is a device scratch double. */
int launch_frame(cudaStream_t s, const Grid& g, const Fields& f, int mode, int a, int b, double* vacc,
                 double* vframe);
/** One launch of the initial guess at time *d_time + tadd: the reference's
 * linear rule, or (quadratic != 0) quadratic-in-time extrapolation from the
 * last three solutions (zprev2 the oldest, unused by the linear rule), which
 * falls back to the linear rule until three exist. */
int launch_guess(cudaStream_t s, double* z, double* zprev, double* zprev2, int n, GuessHist* h,
                 const double* d_time, double tadd, int quadratic, int* err);

/** Gas-layer update (gas_layer::update, gas_layer.cc:36-46) as one CTA.
 * Also advances *d_time by dt/2 (fluid_2d.cc:102). */
int launch_gas_update(cudaStream_t s, const GasPrm& gp, const Gas& gs, const double* u, const double* v, int pitch,
                      const double* d_vframe, double dt, double* d_time, double* work, int* err, GasStats* stats);
/** Size in doubles of the work array launch_gas_update needs. */
size_t gas_work_doubles(int m);
/** Initial gas fields (gas_layer_solve.cc:32-53). */
int launch_gas_init(cudaStream_t s, const GasPrm& gp, const Gas& gs, double h0, double V);
/** Standalone tridiagonal solve (tri_solve::solve_lapack replacement). */
int launch_tri_solve(cudaStream_t s, int n, double* a, double* b, double* c, double* d, int* d_pivoted);

}  // namespace vdi
