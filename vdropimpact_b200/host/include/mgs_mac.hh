// The MAC projection system (mgs_mac.hh:15-74): the 5-point Laplacian of the
// reference on an m x n cell grid, solved on the device.
#ifndef VDI_HOST_MGS_MAC_HH
#define VDI_HOST_MGS_MAC_HH

#include "mgs_common.hh"
#include "tgmg.hh"

struct mgs_mac : public mgs_common {
    const double xxsp;
    const double yysp;
    double acc;
    /** The test constructor (mgs_mac.cc:23-27): grid spacings and source b. */
    mgs_mac(int m_, int n_, double dx, double dy, double* b);
    inline void solve_v_cycle(double t) {
        initial_guess(t);
        solve_v_cycle();
    }
    void solve_v_cycle();
    inline void failure() { fatal_error("Multigrid routine for MAC projection failed", 1); }
    int vdi_kind() const { return VDI_MG_MAC; }
    double vdi_c1() const { return dx_; }
    double vdi_c2() const { return dy_; }
    int vdi_x_sym() const { return 0; }
    tgmg<mgs_mac, double, double> mg;
    private:
        double dx_, dy_;
};

#endif
