// The shared part of the multigrid problem classes (mgs_common.hh:10-56):
// the solution array, the time-extrapolation history and the statistics.
#ifndef VDI_HOST_MGS_COMMON_HH
#define VDI_HOST_MGS_COMMON_HH

#include "common.hh"
#include "tgmg_predict.hh"

struct mgs_common {
    const int m;
    const int n;
    const int mn;
    int scount;
    /** The TGMG problem-class flags (mgs_common.hh:19-26): no periodic
     * direction, the default Gauss-Seidel mode. */
    static const bool x_prd = false;
    static const bool y_prd = false;
    static const char gs_mode = 0;
    double t_prev;
    double t0;
    double* const z_prev;
    double* const z;
    mgs_common(int m_, int n_);
    ~mgs_common();
    /** Linear extrapolation in time from the last two solutions
     * (mgs_common.cc:17-50). */
    void initial_guess(double t);
    inline void reset_counters() {
        wc_time = 0;
        tp.avg_iters(true);
    }
    /** Wall-clock seconds spent in solves. */
    double wc_time;
    tgmg_predict tp;
};

#endif
