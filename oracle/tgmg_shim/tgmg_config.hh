// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// Clean-room stand-in for the absent TGMG configuration header
// (vdropimpact Makefile.dep:63-64 names ../tgmg/tgmg_config.hh). The real
// TGMG source is not available; these constants belong to this shim only.
#ifndef VDI_ORACLE_TGMG_CONFIG_HH
#define VDI_ORACLE_TGMG_CONFIG_HH

#include <cstdlib>

/** Maximum number of V-cycles one solve_v_cycle() call may take. */
const int tgmg_max_vcycles=400;
/** Gauss-Seidel sweeps before / after the coarse-grid correction. */
const int tgmg_nu1=2,tgmg_nu2=2;
/** Coarsening stops once a level has at most this many points; that level
 * is solved directly with a dense LU factorisation. */
const int tgmg_coarse_max=256;

/** Relative residual tolerance ||b-Az||_2 <= rtol*||b||_2 that ends a solve.
 * It defaults to 1e-10 and can be overridden with the VDI_MG_RTOL environment
 * variable or tgmg_set_rtol(). */
inline double& tgmg_rtol_ref() {
    static double rtol=-1;
    if(rtol<0) {
        const char* e=getenv("VDI_MG_RTOL");
        rtol=e?atof(e):1e-10;
    }
    return rtol;
}
inline void tgmg_set_rtol(double r) {tgmg_rtol_ref()=r;}

#endif
