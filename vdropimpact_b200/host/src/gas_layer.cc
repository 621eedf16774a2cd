// Host side of the gas layer: restart records (gas_layer.hh:38-45,
// gas_layer_solve.cc:313-331) and the profile outputs
// (gas_layer_solve.cc:258-308), byte-compatible with the reference's.
#include "gas_layer.hh"

#include <cstring>

#include <cuda_runtime.h>

#include "common.hh"

gas_layer::gas_layer(int m_, double ax_, double bx_, double Vframe_)
    : m(m_), me(m_ + 1), ml(m_ + 4), ax(ax_), bx(bx_), dx((bx_ - ax_) / m_), Vframe(Vframe_), p(new double[me]()),
      tau(new double[ml]()), p_old(new double[me]()), tau_old(new double[ml]()), sim_(NULL) {}

void gas_layer::update(double t, double dt) {
    if (sim_ == NULL) fatal_error("gas_layer::update: the gas layer belongs to no simulation", 1);
    // the device keeps p_old and tau_old, computes the new fields and applies
    // the shear-stress boundary conditions in one pass
    calc_p_and_tau(t, dt);
}

gas_layer::~gas_layer() {
    delete[] tau_old;
    delete[] p_old;
    delete[] tau;
    delete[] p;
}

void gas_layer::apply_tau_bc() {
    tau[0] = -tau[3];
    tau[1] = -tau[2];
    tau[ml - 2] = -tau[ml - 3];
    tau[ml - 1] = -tau[ml - 4];
}

void gas_layer::load_restart(double time, FILE* inf) {
    safe_fread(&Vframe, sizeof(double), 1, inf, "Vframe");
    load_restart_internal(time, inf);
}

void gas_layer::save_restart(FILE* outf) {
    fwrite(&Vframe, sizeof(double), 1, outf);
    save_restart_internal(outf);
}

gas_layer_solve::gas_layer_solve(int m_, double ax_, double bx_, double R_, double V_, double h0_)
    : gas_layer(m_, ax_, bx_, V_), R(R_), V(V_), h0(h0_), h(new double[m_]()), ht(new double[m_]()),
      fbd(new double[m_]()), pg(new double[m_ + 1]()), fm(NULL), fb(NULL) {}

void gas_layer_solve::init_fields() {
    if (sim_ == NULL) fatal_error("gas_layer::init_fields: the gas layer belongs to no simulation", 1);
    vdi_check(vdi_gas_init_fields(sim_), "vdi_gas_init_fields");
    pull();
}

void gas_layer_solve::calc_p_and_tau(double /*t*/, double dt) {
    vdi_check(vdi_gas_update(sim_, dt), "vdi_gas_update");
    pull();
}

void gas_layer_solve::pull() {
    vdi_check(vdi_sim_synchronize(sim_), "vdi_sim_synchronize");
    // device arrays by vdi_sim_device_field index, with their host copies
    struct { int which; double* host; int count; } arr[] = {
        {5, p, me}, {9, p_old, me}, {10, tau, ml}, {11, tau_old, ml},
        {3, h, m}, {12, ht, m}, {13, fbd, m}, {4, pg, me}};
    for (auto& a : arr) {
        double* d = NULL;
        size_t count = 0;
        vdi_check(vdi_sim_device_field(sim_, a.which, &d, &count), "vdi_sim_device_field");
        if (count != size_t(a.count)) fatal_error("gas_layer: device array of unexpected size", 1);
        cudaError_t e = cudaMemcpy(a.host, d, count * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) fatal_error(cudaGetErrorString(e), 1);
    }
}

gas_layer_solve::~gas_layer_solve() {
    delete[] pg;
    delete[] fbd;
    delete[] ht;
    delete[] h;
}

void gas_layer_solve::load_restart_internal(double time, FILE* inf) {
    safe_fread(p, sizeof(double), me, inf, "p array");
    safe_fread(tau + 2, sizeof(double), m, inf, "tau array");
    apply_tau_bc();
    safe_fread(h, sizeof(double), m, inf, "h array");
    safe_fread(ht, sizeof(double), m, inf, "ht array");
    safe_fread(pg, sizeof(double), me, inf, "pg array");
    // the boundary flux is not part of the record; the next update sets it
    memset(fbd, 0, m * sizeof(double));
}

void gas_layer_solve::save_restart_internal(FILE* outf) {
    fwrite(p, sizeof(double), me, outf);
    fwrite(tau + 2, sizeof(double), m, outf);
    fwrite(h, sizeof(double), m, outf);
    fwrite(ht, sizeof(double), m, outf);
    fwrite(pg, sizeof(double), me, outf);
}

void gas_layer_solve::output_profile(const char* filename, float* buf, int sn, double ay, int fld) {
    char* bufc = reinterpret_cast<char*>(buf);
    sprintf(bufc, fld == 0 ? "%s/height.%d" : (fld == 1 ? "%s/fbd.%d" : "%s/pg.%d"), filename, sn);
    FILE* outf = safe_fopen(bufc, "wb");
    int l = fld == 2 ? me : m;
    float* bp = buf + 1;
    *buf = l;
    for (int i = 0; i < l; i++) *(bp++) = ax + (i + (fld == 2 ? 0 : 0.5)) * dx;
    fwrite(buf, sizeof(float), l + 1, outf);
    *buf = ay;
    bp = buf + 1;
    const double* hp = fld == 0 ? h : (fld == 1 ? fbd : pg);
    for (int i = 0; i < l; i++) *(bp++) = hp[i];
    fwrite(buf, sizeof(float), l + 1, outf);
    fclose(outf);
}

void gas_layer_solve::output_profile_double(const char* filename, float* buf, int sn, int fld) {
    char* bufc = reinterpret_cast<char*>(buf);
    sprintf(bufc, fld == 0 ? "%s/hfull.%d" : (fld == 1 ? "%s/fbdfull.%d" : "%s/pgfull.%d"), filename, sn);
    FILE* outf = safe_fopen(bufc, "wb");
    int l = fld == 2 ? me : m;
    fwrite(&l, sizeof(int), 1, outf);
    fwrite(&ax, sizeof(double), 1, outf);
    fwrite(&bx, sizeof(double), 1, outf);
    fwrite(fld == 0 ? h : (fld == 1 ? fbd : pg), sizeof(double), l, outf);
    fclose(outf);
}
