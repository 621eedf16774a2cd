// The multigrid solver object of the reference's problem classes
// (tgmg<S,double,double>, used as msu.mg in mg_test.cc:20-45 and
// mgs_mac.hh:54-72), over the device multigrid of include/vdi.h. The problem
// class S names its system through vdi_kind(), vdi_c1(), vdi_c2() and
// vdi_x_sym(); b and z are host arrays that each call copies to and from the
// device. solve_v_cycle stops at ||b - A z|| <= rtol ||b|| with rtol 1e-10
// (VDI_MG_RTOL overrides it).
#ifndef VDI_HOST_TGMG_HH
#define VDI_HOST_TGMG_HH

#include "tgmg_predict.hh"
#include "vdi.h"

/** The absolute accuracy scale of tgmg_accuracy(scale, fac), the value the
 * problem classes keep in their acc member (mgs_mac.cc:11, mgs_fem.cc:14,
 * visco_impl.cc:12): scale * fac * machine epsilon. The device solves stop on
 * the relative residual instead (rtol above). */
inline double tgmg_accuracy(double scale, double fac) { return scale * fac * 2.220446049250313e-16; }

/** The non-template part: device arrays and the C-ABI calls. */
class vdi_tgmg_core {
    public:
        vdi_tgmg_core(int kind, int m, int n, double* b, double* z);
        ~vdi_tgmg_core();
        void setup(double c1, double c2, int x_sym);
        void clear_z();
        bool solve_v_cycle(tgmg_predict& tp);
        void v_cycle();
        void residual(double* r);
        void output(const char* filename, double* data, double ax, double dx, double ay, double dy);
        void output_res(const char* filename, double ax, double dx, double ay, double dy);
        void output_b(const char* filename, double ax, double dx, double ay, double dy) {
            output(filename, b, ax, dx, ay, dy);
        }
        void output_z(const char* filename, double ax, double dx, double ay, double dy) {
            output(filename, z, ax, dx, ay, dy);
        }
        const int kind, m, n, mn;
        double* const b;
        double* const z;
    private:
        vdi_mg* h;
        double *d_b, *d_z;
        void push();
        void pull();
};

template<class S, class V, class M>
class tgmg : public vdi_tgmg_core {
    public:
        tgmg(S& sys_, V* b_, V* z_) : vdi_tgmg_core(sys_.vdi_kind(), sys_.m, sys_.n, b_, z_), sys(sys_) {}
        /** Builds the device hierarchy for the system's current coefficients. */
        void setup() { vdi_tgmg_core::setup(sys.vdi_c1(), sys.vdi_c2(), sys.vdi_x_sym()); }
    private:
        S& sys;
};

#endif
