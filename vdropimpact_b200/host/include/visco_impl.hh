// The implicit viscous system of one velocity component (visco_impl.hh:15-56)
// bound to a fluid_2d, whose host src array is its right-hand side.
#ifndef VDI_HOST_VISCO_IMPL_HH
#define VDI_HOST_VISCO_IMPL_HH

#include "mgs_common.hh"
#include "tgmg.hh"

class fluid_2d;

struct visco_impl : public mgs_common {
    const bool x_sym;
    const bool horizontal_vel;
    double acc;
    double vfx, vfy;
    visco_impl(fluid_2d& f, bool horizontal_vel_);
    /** Rebuilds the hierarchy when vfx changed (visco_impl.cc:21-39), then
     * extrapolates the guess in time and solves. */
    void setup_and_solve(double vfx_, double vfy_, double t);
    int vdi_kind() const { return horizontal_vel ? VDI_MG_VISC_U : VDI_MG_VISC_V; }
    double vdi_c1() const { return vfx; }
    double vdi_c2() const { return vfy; }
    int vdi_x_sym() const { return x_sym ? 1 : 0; }
    tgmg<visco_impl, double, double> mg;
};

#endif
