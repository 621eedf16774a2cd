// V-cycle statistics of the multigrid solves, with the two calls the
// reference makes on its tgmg_predict (avg_iters, vcount_extra;
// fluid_2d.cc:66-85, mgs_common.hh:47-55).
#ifndef VDI_HOST_TGMG_PREDICT_HH
#define VDI_HOST_TGMG_PREDICT_HH

struct tgmg_predict {
    /** Solves and V-cycles since the last reset. */
    int nsolves, nvcycles;
    tgmg_predict() : nsolves(0), nvcycles(0) {}
    inline void record(int vcycles) {
        nsolves++;
        nvcycles += vcycles;
    }
    inline double avg_iters(bool reset = false) {
        double a = nsolves > 0 ? double(nvcycles) / nsolves : 0.;
        if (reset) nsolves = nvcycles = 0;
        return a;
    }
    inline int vcount_extra() { return nvcycles; }
};

#endif
