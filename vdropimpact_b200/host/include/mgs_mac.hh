// The MAC projection system (mgs_mac.hh:15-74): the 5-point Laplacian of the
// reference on an m x n cell grid, solved on the device.
#ifndef VDI_HOST_MGS_MAC_HH
#define VDI_HOST_MGS_MAC_HH

#include "mgs_common.hh"
#include "tgmg.hh"

class fluid_2d;

struct mgs_mac : public mgs_common {
    const double xxsp;
    const double yysp;
    /** -1 / diagonal for the six kinds of cell (interior or side column
     * crossed with bottom, middle or top row), as inv_cc uses them. */
    const double cc0, cc1, cc2, cc3, cc4, cc5;
    double acc;
    /** Bound to a simulation (mgs_mac.cc:8-15): its spacings, and its src
     * array as the source. */
    mgs_mac(fluid_2d& f);
    /** The test constructor (mgs_mac.cc:23-27): grid spacings and source b. */
    mgs_mac(int m_, int n_, double dx, double dy, double* b);
    // The TGMG problem-class stencil (mgs_mac.hh:25-50), on the host arrays:
    // the 5-point Laplacian with xxsp, yysp couplings. A neighbour beyond a
    // side or the top drops out (Neumann); the bottom row keeps its coupling
    // out of the grid on the diagonal with the ghost reflection of the
    // Dirichlet condition (-3 yysp in all).
    inline double a_dl(int, int) { return 0; }
    inline double a_dr(int, int) { return 0; }
    inline double a_ul(int, int) { return 0; }
    inline double a_ur(int, int) { return 0; }
    inline double a_dc(int, int ij) { return row_kind(ij) > 0 ? yysp : 0; }
    inline double a_uc(int, int ij) { return row_kind(ij) < 2 ? yysp : 0; }
    inline double a_cl(int i, int) { return i > 0 ? xxsp : 0; }
    inline double a_cr(int i, int) { return i < m - 1 ? xxsp : 0; }
    inline double a_cc(int i, int ij) {
        int r = row_kind(ij);
        return (side_column(i) ? -xxsp : -2 * xxsp) + (r == 0 ? -3 * yysp : (r == 1 ? -2 * yysp : -yysp));
    }
    inline double inv_cc(int i, int ij, double v) {
        int r = row_kind(ij);
        double c = side_column(i) ? (r == 0 ? cc3 : (r == 1 ? cc4 : cc5)) : (r == 0 ? cc0 : (r == 1 ? cc1 : cc2));
        return v * c;
    }
    /** The off-diagonal part of A z at (i, ij). */
    inline double mul_a(int i, int ij) {
        const double* w = z + ij;
        double xs = i == 0 ? w[1] : (i < m - 1 ? w[-1] + w[1] : w[-1]);
        int r = row_kind(ij);
        double ys = r == 0 ? w[m] : (r == 1 ? w[-m] + w[m] : w[-m]);
        return xxsp * xs + yysp * ys;
    }
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
        /** 0 bottom row, 1 middle rows, 2 top row. */
        inline int row_kind(int ij) const { return ij < m ? 0 : (ij < mn - m ? 1 : 2); }
        inline bool side_column(int i) const { return i == 0 || i == m - 1; }
};

#endif
