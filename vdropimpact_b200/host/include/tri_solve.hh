// A tridiagonal system with the interface of the reference's tri_solve
// (tri_solve.hh:1-24): public host arrays a (sub-diagonal, a[0] unused),
// b (diagonal), c (super-diagonal, c[m-1] unused) and d (right-hand side,
// overwritten with the solution). Both solve routines run on the device
// (vdi_tri_solve: cyclic reduction, partial pivoting where a row is not
// diagonally dominant); solve_lapack exits on a singular system as the
// reference does (tri_solve.cc:29-32).
#ifndef VDI_HOST_TRI_SOLVE_HH
#define VDI_HOST_TRI_SOLVE_HH

class tri_solve {
    public:
        int m;
        double* const a;
        double* const b;
        double* const c;
        double* const d;
        tri_solve(int m_);
        ~tri_solve();
        void solve();
        void solve_lapack();
    private:
        double* dev;
};

#endif
