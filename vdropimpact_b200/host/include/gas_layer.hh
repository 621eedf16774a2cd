// The gas layer of a B200 simulation, with the public interface of the
// reference's gas_layer (gas_layer.hh:11-60) and gas_layer_solve
// (gas_layer_solve.hh). The arrays are host copies of the device state that
// fluid_2d::sync_fields() refreshes; the update itself runs on the device as
// part of fluid_2d::step_forward.
#ifndef VDI_HOST_GAS_LAYER_HH
#define VDI_HOST_GAS_LAYER_HH

#include <cstdio>

#include "fields.hh"
#include "vdi.h"

class gas_layer {
    public:
        /** The number of grid cells, pressure nodes and ghosted shear-stress
         * entries. */
        const int m, me, ml;
        /** The horizontal extent and the grid spacing. */
        const double ax, bx, dx;
        /** The frame velocity. */
        double Vframe;
        /** Liquid pressure at the nodes, shear stress with two ghost entries on
         * each side, and their values at the previous step. */
        double* const p;
        double* const tau;
        double* const p_old;
        double* const tau_old;
        gas_layer(int m_, double ax_, double bx_, double Vframe_);
        virtual ~gas_layer();
        /** gas_layer::update (gas_layer.cc:38-48): keeps the previous
         * pressure and shear stress, computes new ones from the liquid state
         * and applies the shear-stress boundary conditions. It runs on the
         * device simulation this layer belongs to, reading the device copy of
         * the liquid velocity, and then refreshes the host arrays. */
        void update(double t, double dt);
        /** gas_layer_solve::init_fields (gas_layer_solve.cc:32-53). */
        virtual void init_fields() = 0;
        /** Where the liquid fields live (gas_layer_solve.hh:72). The device
         * update reads the device copy; the pointer is kept for callers. */
        virtual void set_field_pointer(field* fm_) = 0;
        /** The device simulation whose gas layer this is (fluid_2d sets it;
         * no reference counterpart). */
        void attach(vdi_sim* s) { sim_ = s; }
        /** Copies the device's gas-layer arrays into the host arrays. */
        virtual void pull() = 0;
        /** Reads Vframe and the model's fields from a restart file
         * (gas_layer.hh:38-45). */
        void load_restart(double time, FILE* inf);
        void save_restart(FILE* outf);
        virtual void output_profile(const char* filename, float* buf, int sn, double ay, int fld) {}
        virtual void output_profile_double(const char* filename, float* buf, int sn, int fld) {}
    protected:
        virtual void calc_p_and_tau(double t, double dt) = 0;
        virtual void load_restart_internal(double time, FILE* inf) = 0;
        virtual void save_restart_internal(FILE* outf) = 0;
        /** tau = 0 at both ends by odd reflection (gas_layer.cc:25-30). */
        void apply_tau_bc();
        vdi_sim* sim_;
};

/** The model gas layer (gas_layer_model in a .cfg). */
class gas_layer_solve : public gas_layer {
    public:
        /** Drop radius, speed and initial height of the model. */
        const double R, V, h0;
        /** Interface height, its time derivative, the boundary flux and the
         * gas pressure relative to ambient. */
        double* const h;
        double* const ht;
        double* const fbd;
        double* const pg;
        gas_layer_solve(int m_, double ax_, double bx_, double R_, double V_, double h0_);
        ~gas_layer_solve();
        void init_fields();
        void set_field_pointer(field* fm_) {
            fm = fm_;
            fb = fm_ - ml;
        }
        void pull();
        /** Gnuplot binary profile of h (fld 0), fbd (1) or pg (2)
         * (gas_layer_solve.cc:258-282). */
        void output_profile(const char* filename, float* buf, int sn, double ay, int fld);
        /** The same at full precision (gas_layer_solve.cc:290-308). */
        void output_profile_double(const char* filename, float* buf, int sn, int fld);
    protected:
        /** The gas-layer update on the device (vdi_gas_update), then pull(). */
        void calc_p_and_tau(double t, double dt);
        void load_restart_internal(double time, FILE* inf);
        void save_restart_internal(FILE* outf);
    private:
        /** The liquid's (0,0) cell and the row below it. */
        field* fm;
        field* fb;
};

#endif
