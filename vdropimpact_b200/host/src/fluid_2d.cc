// fluid_2d over a B200 simulation: construction, stepping and the frame loop
// (fluid_2d.cc:14-89), and the output and restart routines
// (fluid_2d_sio.cc:14-224) on host copies of the device state.
#include "fluid_2d.hh"

#include <cstdlib>
#include <cstring>
#include <sys/stat.h>
#include <vector>

#include <cuda_runtime.h>

fluid_2d::fluid_2d(const char* infile)
    : fileinfo(infile), mn(m * n), me(m + 1), ne(n + 1), ml(m + 4), dx((bx - ax) / m), dy((by - ay) / n),
      xsp(1. / dx), ysp(1. / dy), xxsp(xsp * xsp), yysp(ysp * ysp),
      dt_reg(implicit_visc ? dx * tmult : dx * dx * rho * muinv * tmult * 0.25),
      fbase(new field[ml * (n + 4)]()), fm(fbase + 2 * ml + 2), tm(new double[2 * ntrace + 2]()), src(new double[me * ne]()),
      s_bc(src + mn), time(0.), f_num(0), S(NULL), buf(new float[m > 123 ? m + 5 : 128]) {
    vdi_check(vdi_sim_create(&params, NULL, &S), "vdi_sim_create");
    vdi_check(vdi_sim_use_graph(S, 1), "vdi_sim_use_graph");
    gl->attach(S);
    gl->set_field_pointer(fm);
}

void fluid_2d::init_tracers() {
    vdi_check(vdi_sim_init_tracers(S), "vdi_sim_init_tracers");
    vdi_check(vdi_sim_get_tracers(S, tm, 2L * ntrace), "vdi_sim_get_tracers");
}

void fluid_2d::update_tracers(double dt) {
    vdi_check(vdi_sim_update_tracers(S, dt), "vdi_sim_update_tracers");
    vdi_check(vdi_sim_get_tracers(S, tm, 2L * ntrace), "vdi_sim_get_tracers");
}

void fluid_2d::set_nif_mode(int mode, double w) {
    vdi_check(vdi_sim_set_nif_mode(S, mode, w), "vdi_sim_set_nif_mode");
    vdi_params p;
    vdi_check(vdi_sim_get_params(S, &p), "vdi_sim_get_params");
    nif_mode = p.nif_mode;
    anif = p.nif_a;
    bnif = p.nif_b;
}

fluid_2d::~fluid_2d() {
    vdi_sim_destroy(S);
    delete[] buf;
    delete[] src;
    delete[] tm;
    delete[] fbase;
}

void fluid_2d::init_fields() {
    vdi_check(vdi_sim_init_fields(S), "vdi_sim_init_fields");
    time = 0.;
    f_num = 0;
    sync_fields();
}

void fluid_2d::step_forward(double dt) {
    vdi_check(vdi_sim_step_forward(S, dt, 1), "vdi_sim_step_forward");
    time += dt;
}

void fluid_2d::solve() {
    double t0, t1, t2, adt;
    int l = timestep_select(t_end / nframes, adt);
    if (f_num == 0) {
        write_files(0);
        puts("# Output frame 0");
    }
    vdi_stats st;
    vdi_check(vdi_sim_stats(S, &st, 1), "vdi_sim_stats");
    long solves[4] = {0, 0, 0, 0}, vcycles[4] = {0, 0, 0, 0};
    t0 = wtime();
    for (int k = f_num + 1; k <= nframes; k++) {
        // the frame's l steps run as graph replays; the call returns after
        // the device-side checks of the last one
        vdi_check(vdi_sim_step_forward(S, adt, l), "vdi_sim_step_forward");
        for (int j = 0; j < l; j++) time += adt;
        t1 = wtime();
        write_files(k);
        t2 = wtime();
        vdi_check(vdi_sim_stats(S, &st, 1), "vdi_sim_stats");
        for (int q = 0; q < 4; q++) {
            solves[q] += st.solves[q];
            vcycles[q] += st.vcycles[q];
        }
        auto avg = [&](int q) { return solves[q] > 0 ? double(vcycles[q]) / solves[q] : 0.; };
        if (mr_time_output) {
            // solver wall-clock times are not measured on the device path
            printf("%d %d %.8g %.8g  %ld %.8g %ld %.8g", k, l, t1 - t0, t2 - t1, st.vcycles[0], 0., st.vcycles[1],
                   0.);
            if (!implicit_visc) printf("  %.8g %.8g\n", 0., 0.);
            else printf(" %ld %.8g %ld %.8g  %.8g %.8g\n", st.vcycles[2], 0., st.vcycles[3], 0., 0., 0.);
        } else {
            printf("# Output frame %d [%d, %.8g s, %.8g s] {MAC %.2f, FEM %.2f", k, l, t1 - t0, t2 - t1, avg(0),
                   avg(1));
            if (!implicit_visc) puts("}");
            else printf(", VX %.2f, VY %.2f}\n", avg(2), avg(3));
        }
        t0 = t2;
    }
}

void fluid_2d::sync_fields() {
    const int tot = ml * (n + 4);
    std::vector<double> u(tot), v(tot), p(tot);
    gas_layer_solve* g = static_cast<gas_layer_solve*>(gl);
    std::vector<double> tau(ml);
    vdi_state s;
    s.u = u.data();
    s.v = v.data();
    s.p = p.data();
    s.gp = g->p;
    s.tau = tau.data();
    s.h = g->h;
    s.fbd = g->fbd;
    s.pg = g->pg;
    s.ht = g->ht;
    vdi_check(vdi_sim_get_state(S, &s), "vdi_sim_get_state");
    vdi_check(vdi_sim_get_tracers(S, tm, 2L * ntrace), "vdi_sim_get_tracers");
    for (int k = 0; k < tot; k++) {
        fbase[k].u = u[k];
        fbase[k].v = v[k];
        fbase[k].p = p[k];
    }
    memcpy(g->tau, tau.data(), ml * sizeof(double));
    g->Vframe = s.Vframe;
    time = s.time;
    double* d_src = NULL;
    size_t count = 0;
    vdi_check(vdi_sim_device_field(S, 8, &d_src, &count), "vdi_sim_device_field");
    cudaError_t e = cudaMemcpy(src, d_src, count * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) fatal_error(cudaGetErrorString(e), 1);
}

void fluid_2d::push_fields() {
    const int tot = ml * (n + 4);
    std::vector<double> u(tot), v(tot), p(tot);
    for (int k = 0; k < tot; k++) {
        u[k] = fbase[k].u;
        v[k] = fbase[k].v;
        p[k] = fbase[k].p;
    }
    gas_layer_solve* g = static_cast<gas_layer_solve*>(gl);
    vdi_state s;
    s.time = time;
    s.Vframe = g->Vframe;
    s.u = u.data();
    s.v = v.data();
    s.p = p.data();
    s.gp = g->p;
    s.tau = g->tau;
    s.h = g->h;
    s.fbd = g->fbd;
    s.pg = g->pg;
    s.ht = g->ht;
    vdi_check(vdi_sim_set_state(S, &s), "vdi_sim_set_state");
    vdi_check(vdi_sim_set_tracers(S, tm, 2L * ntrace), "vdi_sim_set_tracers");
}

void fluid_2d::load_restart(int sn) {
    FILE* inf = odir_open("res", sn, "rb");
    safe_fread(&time, sizeof(double), 1, inf, "simulation time");
    f_num = sn;
    std::vector<double> lbuf(3 * ml);
    field* fp = fbase;
    for (int j = 0; j < n + 4; j++) {
        safe_fread(lbuf.data(), sizeof(double), 3 * ml, inf, "primary fields");
        double* lp = lbuf.data();
        for (int i = 0; i < ml; i++) (fp++)->unpack(lp);
    }
    safe_fread(tm, sizeof(double), ntrace << 1, inf, "tracer information");
    gl->load_restart(time, inf);
    fclose(inf);
    push_fields();
}

bool fluid_2d::restart_exists(int sn) {
    char* bufc = reinterpret_cast<char*>(buf);
    sprintf(bufc, "%s/res.%d", filename, sn);
    struct stat st;
    return stat(bufc, &st) == 0;
}

void fluid_2d::load_last_restart() {
    if (restart_freq == 0) puts("# Restart frequency not set, starting from frame 0");
    if (restart_exists(restart_freq)) {
        int lr = restart_freq;
        while (restart_exists(lr + restart_freq)) {
            lr += restart_freq;
            if (lr >= nframes) {
                fputs("# Final restart file found; nothing to do\n", stderr);
                exit(1);
            }
        }
        printf("# Starting from restart file at frame %d\n", lr);
        load_restart(lr);
        return;
    } else puts("# No restart file found, starting from frame 0");
    init_fields();
}

void fluid_2d::save_restart(int sn) {
    sync_fields();
    FILE* outf = odir_open("res", sn, "wb");
    fwrite(&time, sizeof(double), 1, outf);
    std::vector<double> lbuf(3 * ml);
    field* fp = fbase;
    for (int j = 0; j < n + 4; j++) {
        double* lp = lbuf.data();
        for (int i = 0; i < ml; i++) (fp++)->pack(lp);
        fwrite(lbuf.data(), sizeof(double), 3 * ml, outf);
    }
    fwrite(tm, sizeof(double), ntrace << 1, outf);
    gl->save_restart(outf);
    fclose(outf);
}

void fluid_2d::write_files(int k) {
    sync_fields();
    if (fflags & 1) output("u", 0, k, true);
    if (fflags & 2) output("v", 1, k, true);
    if (fflags & 4) output("p", 2, k);
    if (fflags & 8) output("pb", 3, k);
    if (fflags & 16) output_pbase_full(k);
    if (fflags & 32) output("w", 4, k);
    if (fflags & 64) gl->output_profile(filename, buf, k, ay, 0);
    if (fflags & 128) gl->output_profile(filename, buf, k, ay, 1);
    if (fflags & 256) gl->output_profile(filename, buf, k, ay, 2);
    if (fflags & 512) gl->output_profile_double(filename, buf, k, 0);
    if (fflags & 1024) gl->output_profile_double(filename, buf, k, 1);
    if (fflags & 2048) gl->output_profile_double(filename, buf, k, 2);
    if (ntrace > 0) output_tracers(k);
    if (restart_freq > 0 && k > 0 && k % restart_freq == 0) save_restart(k);
}

void fluid_2d::output_tracers(const int sn) {
    // fluid_2d_sio.cc:121-145: the 2*ntrace coordinates as floats
    FILE* outf = odir_open("trace", sn, "wb");
    const int tot = ntrace << 1;
    for (int j = 0; j < tot; j += 128) {
        const int c = tot - j < 128 ? tot - j : 128;
        for (int q = 0; q < c; q++) buf[q] = float(tm[j + q]);
        fwrite(buf, sizeof(float), c, outf);
    }
    fclose(outf);
}

void fluid_2d::output_pbase_full(const int sn) {
    FILE* outf = odir_open("pbfull", sn, "wb");
    fwrite(&me, sizeof(int), 1, outf);
    fwrite(&ax, sizeof(double), 1, outf);
    fwrite(&bx, sizeof(double), 1, outf);
    std::vector<double> pr(me);
    for (int o = 0; o < me; o++) pr[o] = fm[o].p;
    fwrite(pr.data(), sizeof(double), me, outf);
    fclose(outf);
}

void fluid_2d::output(const char* prefix, const int mode, const int sn, const bool ghost) {
    // the Gnuplot binary matrix of one field (fluid_2d_sio.cc:183-224):
    // cell-centred u, v (with ghosts), nodal p, the bottom row of p, or the
    // nodal vorticity
    bool cen = mode >= 0 && mode <= 1;
    int li = ghost ? ml : (cen ? m : m + 1), lj = mode == 3 ? 1 : (ghost ? n + 4 : (cen ? n : n + 1));
    double disp = (cen ? 0.5 : 0) - (ghost ? 2 : 0);
    FILE* outf = odir_open(prefix, sn, "wb");
    float* bp = buf + 1;
    *buf = li;
    for (int i = 0; i < li; i++) *(bp++) = ax + (i + disp) * dx;
    fwrite(buf, sizeof(float), li + 1, outf);
    field* fr = ghost ? fbase : fm;
    for (int j = 0; j < lj; j++, fr += ml) {
        field* fp = fr;
        *buf = ay + (j + disp) * dy;
        bp = buf + 1;
        for (int i = 0; i < li; i++, fp++) {
            switch (mode) {
                case 0: *(bp++) = fp->u; break;
                case 1: *(bp++) = fp->v; break;
                case 2:
                case 3: *(bp++) = fp->p; break;
                case 4: *(bp++) = vorticity(fp);
            }
        }
        fwrite(buf, sizeof(float), li + 1, outf);
    }
    fclose(outf);
}
