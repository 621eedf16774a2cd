// Device lift-off search (tt_analysis.cc:97-171): configuration, state and
// launch helpers shared by the simulation and the standalone entry point.
#pragma once

#include <cuda_runtime.h>

namespace vdi {

constexpr int LIFTOFF_MAX_M = 8192;     // gas-layer cells one CTA analyses (3 doubles each in shared memory)
constexpr int LIFTOFF_MAX_CUT = 64;     // Gaussian half-width in cells (dx >= glen / 9.1)

struct LiftoffCfg {
    int m, mode, every, cut;
    double ax, dx;                      // cell centres x_i = ax + (i + 1/2) dx, stored as float32
    double R, V, h_ev;
    double w[2 * LIFTOFF_MAX_CUT + 1];  // normalised Gaussian weights, w[cut + j] for offset j
};

/** The search state (tt_analysis.cc:94-96, 149-163), in device memory. */
struct LiftoffState {
    long counter;          // steps seen since the last reset
    long count;            // states analysed
    long gimin;            // index of the state with the global minimum
    double gfmin, gxmin;   // the global minimum height and its position
    double tmin0_ev;       // evanescent-field time origin
    double last_x, last_f; // minimum of the last analysed state
    double interval;       // time between analysed states
    int hsearch, efield;
};

int liftoff_config(int m, double ax, double dx, int mode, int every, double R, double V, LiftoffCfg* c);
int liftoff_reset_async(cudaStream_t s, LiftoffState* st);
int liftoff_launch(cudaStream_t s, const double* h, const LiftoffCfg& c, LiftoffState* st, double2* hist, long cap,
                   double dt);

}  // namespace vdi
