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
    // The TGMG problem-class stencil (visco_impl.hh:28-53), on the host
    // arrays: I - vfx d_xx - vfy d_yy with a Neumann top and sides; the bottom
    // row and, with x_sym, the axis column carry their ghost reflections on the
    // diagonal (the horizontal velocity is odd about the axis).
    inline double a_dl(int, int) { return 0.; }
    inline double a_dr(int, int) { return 0.; }
    inline double a_ul(int, int) { return 0.; }
    inline double a_ur(int, int) { return 0.; }
    inline double a_dc(int, int ij) { return ij >= m ? -vfy : 0.; }
    inline double a_uc(int, int ij) { return ij < mn - m ? -vfy : 0.; }
    inline double a_cl(int i, int) { return i > 0 ? -vfx : 0.; }
    inline double a_cr(int i, int) { return i < m - 1 ? -vfx : 0.; }
    inline double a_cc(int i, int ij) {
        double xpart = !x_sym || i > 0 ? 2 * vfx : (horizontal_vel ? 3 * vfx : vfx);
        return 1 + xpart + (ij >= m ? 2 * vfy : vfy);
    }
    inline double inv_cc(int i, int ij, double v) { return v / a_cc(i, ij); }
    /** The off-diagonal part of A z at (i, ij). */
    inline double mul_a(int i, int ij) {
        const double* w = z + ij;
        double xs = i > 0 ? (i < m - 1 ? w[1] + w[-1] : w[-1]) : w[1];
        double ys = ij >= m ? (ij < mn - m ? w[m] + w[-m] : w[-m]) : w[m];
        return -vfx * xs - vfy * ys;
    }
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
