// The finite-element projection system (mgs_fem.hh:17-81): the bilinear
// 9-point operator of the reference on an m x n node grid with the Dirichlet
// bottom row, solved on the device.
#ifndef VDI_HOST_MGS_FEM_HH
#define VDI_HOST_MGS_FEM_HH

#include "mgs_common.hh"
#include "tgmg.hh"

class fluid_2d;

struct mgs_fem : public mgs_common {
    /** Spacing ratios and the bilinear element's stencil terms
     * (mgs_fem.cc:8-11): centre fm (and its reciprocal), vertical fey, hey,
     * horizontal fex, hex (the h* halves for edge nodes), corner fc. */
    const double dydx, dxdy, fm, fm_inv, fey, hey, fex, hex, fc;
    double acc;
    /** Bound to a simulation (mgs_fem.cc:8-18): its spacings on the node
     * grid, and its src array as the source. */
    mgs_fem(fluid_2d& f);
    /** The test constructor (mgs_fem.cc:26-30). */
    mgs_fem(int m_, int n_, double dx, double dy, double* b);
    // The TGMG problem-class stencil (mgs_fem.hh:42-57), on the host arrays:
    // the 9-point bilinear finite-element operator on m x n nodes. Nodes on
    // the left, right and top edges carry half the element weight; the bottom
    // row is a Dirichlet row with only its diagonal.
    inline bool bottom(int ij) { return ij < m; }
    inline double a_dl(int i, int ij) { return !bottom(ij) && i > 0 ? fc : 0; }
    inline double a_dr(int i, int ij) { return !bottom(ij) && i < m - 1 ? fc : 0; }
    inline double a_ul(int i, int ij) { return !bottom(ij) && below_top(ij) && i > 0 ? fc : 0; }
    inline double a_ur(int i, int ij) { return !bottom(ij) && below_top(ij) && i < m - 1 ? fc : 0; }
    inline double a_dc(int i, int ij) { return !bottom(ij) ? (inner_column(i) ? fey : hey) : 0; }
    inline double a_uc(int i, int ij) { return !bottom(ij) && below_top(ij) ? (inner_column(i) ? fey : hey) : 0; }
    inline double a_cl(int i, int ij) { return !bottom(ij) && i > 0 ? (below_top(ij) ? fex : hex) : 0; }
    inline double a_cr(int i, int ij) { return !bottom(ij) && i < m - 1 ? (below_top(ij) ? fex : hex) : 0; }
    inline double a_cc(int i, int ij) {
        return (inner_column(i) ? 1 : 0.5) * (inner_row(ij) ? 1 : 0.5) * fm;
    }
    inline double inv_cc(int i, int ij, double v) {
        return (inner_column(i) ? 1 : 2) * (inner_row(ij) ? 1 : 2) * fm_inv * v;
    }
    /** The off-diagonal part of A z at (i, ij); 0 on the Dirichlet bottom
     * row (mgs_fem.cc:32-53). */
    double mul_a(int i, int ij);
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
        inline bool inner_column(int i) const { return i > 0 && i < m - 1; }
        inline bool below_top(int ij) const { return ij < mn - m; }
        inline bool inner_row(int ij) const { return ij >= m && ij < mn - m; }
};

#endif
