// The configuration of a run read from a .cfg file, with the members of the
// reference's fileinfo (fileinfo.hh:16-96). Parsing goes through the C ABI
// (vdi_params_from_cfg, vdi_run_options_from_cfg); errors exit through
// fatal_error as in the reference (fileinfo.cc:11-193).
#ifndef VDI_HOST_FILEINFO_HH
#define VDI_HOST_FILEINFO_HH

#include "gas_layer.hh"
#include "vdi.h"

struct fileinfo {
    public:
        int m;
        int n;
        unsigned int fflags;
        int ntrace;
        int nframes;
        int restart_freq;
        /** The non-inertial frame mode: 0 off, 1 nif_center, 2 nif_range. */
        int nif_mode;
        bool implicit_visc;
        bool x_sym;
        bool mr_time_output;
        double ax;
        const double ay;
        double bx;
        double by;
        double dx;
        double dy;
        double xsp;
        double ysp;
        double mu;
        double muinv;
        double rho;
        double rhoinv;
        double tmult;
        double t_end;
        /** The output directory (the .cfg name with .odr). */
        char* filename;
        gas_layer* gl;
        /** The columns [anif, bnif) whose velocity nif_range averages
         * (fileinfo.hh:84-86, fileinfo.cc:179-191). */
        int anif;
        int bnif;
        fileinfo(const char* infile);
        ~fileinfo();
        /** The parameters in the C-ABI form. */
        vdi_params params;
};

#endif
