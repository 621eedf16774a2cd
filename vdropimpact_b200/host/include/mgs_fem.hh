// The finite-element projection system (mgs_fem.hh:17-81): the bilinear
// 9-point operator of the reference on an m x n node grid with the Dirichlet
// bottom row, solved on the device.
#ifndef VDI_HOST_MGS_FEM_HH
#define VDI_HOST_MGS_FEM_HH

#include "mgs_common.hh"
#include "tgmg.hh"

struct mgs_fem : public mgs_common {
    const double dydx, dxdy, fm;
    double acc;
    /** The test constructor (mgs_fem.cc:26-30). */
    mgs_fem(int m_, int n_, double dx, double dy, double* b);
    inline void solve_v_cycle(double t) {
        initial_guess(t);
        solve_v_cycle();
    }
    void solve_v_cycle();
    inline void failure() { fatal_error("Multigrid routine for finite-element projection failed", 1); }
    int vdi_kind() const { return VDI_MG_FEM; }
    double vdi_c1() const { return dx_; }
    double vdi_c2() const { return dy_; }
    int vdi_x_sym() const { return 0; }
    tgmg<mgs_fem, double, double> mg;
    private:
        double dx_, dy_;
};

#endif
