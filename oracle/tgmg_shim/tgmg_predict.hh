// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// Clean-room stand-in for TGMG's V-cycle statistics helper. The reference
// only calls avg_iters(bool) and vcount_extra() (fluid_2d.cc:66-85,
// mgs_common.hh:47-55); this shim records V-cycles per solve.
#ifndef VDI_ORACLE_TGMG_PREDICT_HH
#define VDI_ORACLE_TGMG_PREDICT_HH

struct tgmg_predict {
    /** Solves and V-cycles recorded since the last reset. */
    int nsolves,nvcycles;
    /** V-cycles taken by the most recent solve. */
    int last;
    tgmg_predict() : nsolves(0), nvcycles(0), last(0) {}
    inline void record(int v) {nsolves++;nvcycles+=v;last=v;}
    /** Average V-cycles per solve; resets the counters when asked to. */
    inline double avg_iters(bool reset=false) {
        double a=nsolves>0?double(nvcycles)/nsolves:0.;
        if(reset) nsolves=nvcycles=0;
        return a;
    }
    /** Total V-cycles since the last reset. */
    inline int vcount_extra() {return nvcycles;}
};

#endif
