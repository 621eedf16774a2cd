// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// The reference calls LAPACK's dgtsv_ (tri_solve.cc:7-9, 28). No system
// LAPACK is installed; SciPy's bundled OpenBLAS exports the same routine as
// scipy_dgtsv_ (32-bit integer interface), so the oracle build forwards to it.
extern "C" {
void scipy_dgtsv_(int* n,int* nrhs,double* dl,double* d,double* du,double* b,int* ldb,int* info);
void dgtsv_(int* n,int* nrhs,double* dl,double* d,double* du,double* b,int* ldb,int* info) {
    scipy_dgtsv_(n,nrhs,dl,d,du,b,ldb,info);
}
}
