// The step driver with the public interface of the reference's fluid_2d
// (fluid_2d.hh:21-142) over a B200 simulation (vdi_sim of include/vdi.h).
//
// step_forward, init_fields and solve run on the device; the frame output
// (write_files and the Gnuplot formats of fluid_2d_sio.cc:140-224) and the
// restart files (fluid_2d_sio.cc:39-119) are byte-compatible with the
// reference's. fbase/fm hold host copies of u, v, p that sync_fields()
// refreshes; the output and restart routines call it themselves. Tracers
// (tm, trace.N files and their restart block) and the non-inertial frame
// run on the device with the rest of the step.
#ifndef VDI_HOST_FLUID_2D_HH
#define VDI_HOST_FLUID_2D_HH

#include <cstdio>

#include "common.hh"
#include "fields.hh"
#include "fileinfo.hh"
#include "vdi.h"

class fluid_2d : public fileinfo {
    public:
        const int mn;
        const int me;
        const int ne;
        const int ml;
        const double dx;
        const double dy;
        const double xsp;
        const double ysp;
        const double xxsp;
        const double yysp;
        const double dt_reg;
        /** Host copy of the primary fields over the ghosted grid. */
        field* const fbase;
        /** The (0,0) cell of fbase. */
        field* const fm;
        /** Tracer positions x0, y0, x1, ... (2*ntrace; host copy of the
         * device's, refreshed by sync_fields). */
        double* const tm;
        /** The host source array of the node grid (me*ne), shared as in the
         * reference (fluid_2d.cc:18-21): the right-hand side of problem
         * objects bound to this fluid_2d. sync_fields() fills it with the
         * device's last FEM source, which is what the reference's shared
         * array holds after a step. */
        double* const src;
        /** src + mn (fluid_2d.cc:18): in the reference the bottom-row terms of
         * the MAC source, which the FEM source then overwrites. */
        double* const s_bc;
        double time;
        int f_num;
        fluid_2d(const char* infile);
        ~fluid_2d();
        void solve();
        void step_forward(double dt);
        void init_fields();
        void load_restart(int sn);
        void load_last_restart();
        void save_restart(int sn);
        void write_files(int k);
        void output(const char* prefix, const int mode, int sn, bool ghost = false);
        void output_pbase_full(int sn);
        void output_tracers(int sn);
        /** fluid_2d::init_tracers (fluid_2d.cc:495-502) on the device tracers,
         * then refreshes tm. */
        void init_tracers();
        /** fluid_2d::update_tracers (fluid_2d.cc:507-526): moves the device
         * tracers by dt with the device velocity, then refreshes tm. */
        void update_tracers(double dt);
        /** Switches the non-inertial frame (fluid_2d.hh:75): mode 0 off, 1 the
         * velocity at the centre, 2 averaged over the columns within w of the
         * axis. The reference declares it without a body. */
        void set_nif_mode(int mode, double w = 0);
        inline int timestep_select(double interval, double& adt) {
            int l = static_cast<int>(interval / dt_reg) + 1;
            adt = interval / l;
            return l;
        }
        inline FILE* odir_open(const char* prefix, int sn, const char* mode) {
            char* bufc = reinterpret_cast<char*>(buf);
            sprintf(bufc, "%s/%s.%d", filename, prefix, sn);
            return safe_fopen(bufc, mode);
        }
        /** Copies u, v, p, the gas-layer arrays and the time from the device
         * into fbase/fm, gl and time. */
        void sync_fields();
        /** The device simulation (for callers of the C ABI). */
        vdi_sim* sim() { return S; }
    private:
        vdi_sim* S;
        float* buf;
        bool restart_exists(int sn);
        /** Copies fbase/fm, gl and time to the device. */
        void push_fields();
        inline double vorticity(field* fp) {
            return 0.5 * (xsp * (fp->v - fp[-1].v + fp[-ml].v - fp[-ml - 1].v) -
                          ysp * (fp->u + fp[-1].u - fp[-ml].u - fp[-ml - 1].u));
        }
};

#endif
