// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// Exercises the members of the drop-in boundary that a driver written
// against the reference's classes calls, and prints every value. The same
// source is compiled twice by oracle/Makefile: against the reference's own
// headers and objects (with the shims of this directory) as _ref/boundary_probe,
// and against the drop-in headers of vdropimpact_b200/host as
// _ref/boundary_probe_b200 (VDI_PROBE_B200 defined). tests/test_gpu_boundary.py
// runs both on the same configuration and compares the outputs.
//
//   boundary_probe <cfg>
//
// Members exercised (reference file:line):
//   TGMG problem-class accessors a_dl..a_ur, a_cc, inv_cc, mul_a of mgs_mac
//     (mgs_mac.hh:25-50), mgs_fem (mgs_fem.hh:42-57, mgs_fem.cc:32-53) and
//     visco_impl (visco_impl.hh:28-53), and the constants cc0..cc5, fm_inv,
//     fey, hey, fex, hex, fc;
//   the flags x_prd, y_prd, gs_mode (mgs_common.hh:19-26);
//   mgs_mac(fluid_2d&), mgs_fem(fluid_2d&) (mgs_mac.cc:8-15, mgs_fem.cc:8-18)
//     and a solve from the simulation's src;
//   fluid_2d::src and s_bc after steps (fluid_2d.cc:18-21, 218-232, 337-377);
//   gas_layer::update(t, dt), init_fields(), set_field_pointer()
//     (gas_layer.cc:38-48, gas_layer_solve.cc:32-53, gas_layer_solve.hh:72);
//   fluid_2d::init_tracers(), update_tracers(dt) (fluid_2d.cc:495-526).
//
// Output: one line per quantity, "name v0 v1 ...", values with %.17g.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fluid_2d.hh"
#include "gas_layer_solve.hh"
#include "mgs_fem.hh"
#include "mgs_mac.hh"
#include "visco_impl.hh"


static void put(const char* name, const double* v, int n) {
    printf("%s", name);
    for (int k = 0; k < n; k++) printf(" %.17g", v[k]);
    putchar('\n');
}

static void put1(const char* name, double v) { put(name, &v, 1); }

/** A deterministic, non-smooth pattern for solution arrays. */
static void pattern(double* z, int n, double a) {
    for (int k = 0; k < n; k++) z[k] = std::sin(a * k + 0.3) + 0.01 * (k % 7);
}

/** Every accessor of a problem class at every point. */
template<class S>
static void accessors(const char* tag, S& s) {
    pattern(s.z, s.mn, 0.7);
    std::vector<double> v;
    for (int ij = 0; ij < s.mn; ij++) {
        int i = ij % s.m;
        double row[12] = {s.a_dl(i, ij), s.a_dc(i, ij), s.a_dr(i, ij), s.a_cl(i, ij), s.a_cc(i, ij),
                          s.a_cr(i, ij), s.a_ul(i, ij), s.a_uc(i, ij), s.a_ur(i, ij), s.inv_cc(i, ij, 1.3),
                          s.mul_a(i, ij), s.inv_cc(i, ij, -0.25)};
        v.insert(v.end(), row, row + 12);
    }
    char name[64];
    snprintf(name, sizeof(name), "%s_stencil", tag);
    put(name, v.data(), int(v.size()));
    double flags[3] = {double(S::x_prd), double(S::y_prd), double(S::gs_mode)};
    snprintf(name, sizeof(name), "%s_flags", tag);
    put(name, flags, 3);
}

int main(int argc, char** argv) {
    if (argc < 2) {
        fputs("usage: boundary_probe <cfg>\n", stderr);
        return 2;
    }
    // problem classes with the test constructors
    {
        std::vector<double> b(7 * 5, 0.);
        mgs_mac s(7, 5, 0.3, 0.2, b.data());
        accessors("mac", s);
        double c[8] = {s.xxsp, s.yysp, s.cc0, s.cc1, s.cc2, s.cc3, s.cc4, s.cc5};
        put("mac_constants", c, 8);
    }
    {
        std::vector<double> b(7 * 6, 0.);
        mgs_fem s(7, 6, 0.3, 0.2, b.data());
        accessors("fem", s);
        double c[9] = {s.dydx, s.dxdy, s.fm, s.fm_inv, s.fey, s.hey, s.fex, s.hex, s.fc};
        put("fem_constants", c, 9);
    }
    fluid_2d f(argv[1]);
    for (int horiz = 0; horiz < 2; horiz++) {
        visco_impl vi(f, horiz != 0);
        vi.vfx = 0.37;
        vi.vfy = 0.52;
        accessors(horiz ? "viscu" : "viscv", vi);
    }

    // the simulation: init, three steps, its shared source array
    f.init_fields();
    double adt;
    f.timestep_select(f.t_end / f.nframes, adt);
    for (int k = 0; k < 3; k++) f.step_forward(adt);
#ifdef VDI_PROBE_B200
    f.sync_fields();
#endif
    put("src_after_steps", f.src, f.me * f.ne);
    put("s_bc_after_steps", f.s_bc, f.m);

    // the tracers: placed with rand() after a fixed seed, moved one step
    if (f.ntrace > 0) {
        srand(12345);
        f.init_tracers();
        put("tracers_init", f.tm, 2 * f.ntrace);
        f.update_tracers(adt);
        put("tracers_moved", f.tm, 2 * f.ntrace);
    }

    // the gas layer on its own: one more update from the current state
    gas_layer_solve* g = dynamic_cast<gas_layer_solve*>(f.gl);
    if (g == NULL) {
        fputs("gas_layer_model required\n", stderr);
        return 2;
    }
    g->set_field_pointer(f.fm);
    g->update(f.time, adt);
    put("gas_p", g->p, g->me);
    put("gas_p_old", g->p_old, g->me);
    put("gas_tau", g->tau, g->ml);
    put("gas_tau_old", g->tau_old, g->ml);
    put("gas_h", g->h, g->m);
    put("gas_pg", g->pg, g->me);
    g->init_fields();
    put("gas_init_h", g->h, g->m);
    put("gas_init_ht", g->ht, g->m);
    put("gas_init_pg", g->pg, g->me);
    put("gas_init_p", g->p, g->me);

    // problem objects bound to the simulation, solving from its src
    {
        mgs_mac s(f);
        double c[8] = {s.xxsp, s.yysp, s.cc0, s.cc1, s.cc2, s.cc3, s.cc4, s.cc5};
        put("mac_f_constants", c, 8);
        for (int ij = 0; ij < s.mn; ij++) f.src[ij] = std::cos(0.01 * ij) * (ij % 13 - 6);
        s.solve_v_cycle();
        put("mac_f_z", s.z, s.mn);
    }
    {
        mgs_fem s(f);
        double c[9] = {s.dydx, s.dxdy, s.fm, s.fm_inv, s.fey, s.hey, s.fex, s.hex, s.fc};
        put("fem_f_constants", c, 9);
        for (int ij = 0; ij < s.mn; ij++) f.src[ij] = ij < s.m ? s.a_cc(ij, ij) * 0.5 : std::sin(0.02 * ij);
        s.solve_v_cycle();
        put("fem_f_z", s.z, s.mn);
    }
    put1("done", 1);
    return 0;
}
