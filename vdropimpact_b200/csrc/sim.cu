// The step driver (fluid_2d, fluid_2d.cc:14-405) over the device kernels,
// and the C ABI declared in include/vdi.h.
#include "step_kernels.hh"
#include "liftoff.hh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

namespace vdi {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

}  // namespace vdi

using namespace vdi;

enum { SOLVER_MAC = 0, SOLVER_FEM = 1, SOLVER_VX = 2, SOLVER_VY = 3 };

struct vdi_sim {
    vdi_params prm{};
    Grid g{};
    GasPrm gp{};
    double dt_reg = 0;
    cudaStream_t s = nullptr, s_gas = nullptr, s_vy = nullptr, s_guess = nullptr;
    bool own_stream = false;
    cudaEvent_t ev_fork = nullptr, ev_gas = nullptr, ev_vy = nullptr, ev_vy_done = nullptr;
    cudaEvent_t ev_adv = nullptr, ev_side = nullptr;   // advection done; side-stream work done
    cudaEvent_t ev_guess = nullptr;                    // the MAC guess done
    std::vector<double*> bufs;
    Fields f{};
    Gas gas{};
    double* gas_work = nullptr;
    double *src_mac = nullptr, *q = nullptr, *q_prev = nullptr;
    double *src_fem = nullptr, *zf = nullptr, *zf_prev = nullptr;
    // third-latest solutions for the quadratic initial guess
    double *q_prev2 = nullptr, *zu_prev2 = nullptr, *zv_prev2 = nullptr, *zf_prev2 = nullptr;
    double *su = nullptr, *sv = nullptr, *zu = nullptr, *zu_prev = nullptr, *zv = nullptr, *zv_prev = nullptr;
    GuessHist* hist = nullptr;   // 4 entries
    double* d_time = nullptr;
    double* d_vframe = nullptr;
    double* d_tm = nullptr;     // tracer positions x0, y0, x1, ... (2 * ntrace)
    double* d_vacc = nullptr;   // the non-inertial frame's velocity of a step
    double* d_time_aside = nullptr;   // clock for a gas-layer update run alone
    double* d_time_start = nullptr;   // the clock at the start of a step (the MAC guess's)
    int* d_err = nullptr;
    GasStats* d_gstats = nullptr;
    MG* mg[4] = {nullptr, nullptr, nullptr, nullptr};
    double vfx_cur = 0, vfy_cur = 0;
    double fem_acc_edge = 0, fem_acc_mid = 0;
    // graph replay of one step
    bool use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    double graph_dt = 0;
    long steps = 0;
    // learned initial guess of the MAC solve
    vdi_unet* unet = nullptr;
    int unet_factor = 0;
    double unet_scale = 0;
    double* unet_r = nullptr;      // residual of the extrapolated guess (m x n)
    double* unet_norm = nullptr;   // its 2-norm
    float *unet_in = nullptr, *unet_out = nullptr;
    // advection stages as one fused kernel (VDI_FUSED_ADVECT=0: four kernels)
    bool fused_advect = true;
    // the viscous guesses on the side stream beside the MAC solve
    // (VDI_VISC_GUESS_SIDE=0: on the viscous solves' own streams)
    bool visc_guess_side = true;
    // lift-off search (tt_analysis.cc:97-171) after every step
    LiftoffCfg lcfg{};
    LiftoffState* d_lift = nullptr;
    double2* d_lhist = nullptr;
    long lcap = 0;
};

namespace {

int alloc_zero(vdi_sim* S, double** p, size_t n) {
    VDI_CUDA(cudaMalloc(p, n * sizeof(double)));
    VDI_CUDA(cudaMemset(*p, 0, n * sizeof(double)));
    S->bufs.push_back(*p);
    return VDI_OK;
}

size_t ghosted(const vdi_sim* S) { return size_t(S->prm.m + 4) * (S->prm.n + 4); }

/** visco_impl::setup_and_solve's re-setup test (visco_impl.cc:26-30). */
int update_visc(vdi_sim* S, double dt) {
    const Grid& g = S->g;
    if (!g.implicit_visc) return VDI_OK;
    double vfx = g.viscfac * g.xxsp * dt, vfy = g.viscfac * g.yysp * dt;
    if (std::fabs(vfx - S->vfx_cur) > 1e2 * 2.220446049250313e-16 * S->vfx_cur || S->vfx_cur == 0) {
        S->vfx_cur = vfx;
        S->vfy_cur = vfy;
        VDI_TRY(mg_set_visc(S->mg[SOLVER_VX], vfx, vfy));
        VDI_TRY(mg_set_visc(S->mg[SOLVER_VY], vfx, vfy));
    }
    return VDI_OK;
}

/** mgs_common::initial_guess (mgs_common.cc:17-50) for one solver, or the
 * quadratic variant when the parameters ask for it, at time *d_time + tadd. */
int guess(vdi_sim* S, cudaStream_t s, int which, double* z, double* zp, double* zp2, int n, double tadd = 0.,
          const double* clock = nullptr) {
    const int quad = S->prm.mg_guess == VDI_GUESS_QUADRATIC || S->prm.mg_guess == VDI_GUESS_LEARNED;
    return launch_guess(s, z, zp, zp2, n, S->hist + which, clock ? clock : S->d_time, tadd, quad, S->d_err);
}

/** Enqueues one fluid_2d::step_forward(dt) (fluid_2d.cc:93-405). */
int enqueue_step(vdi_sim* S, double dt) {
    const Grid& g = S->g;
    cudaStream_t s = S->s;
    const int m = g.m, n = g.n, mn = m * n, nf = (m + 1) * (n + 1);
    int prec = S->prm.mg_precision;
    // The gas layer runs on its own stream, overlapping the advection. The
    // same stream then takes the work that needs neither the advection's
    // output nor the MAC solve, off the main stream's path:
    //  - once the advection has read the ghost cells, the far-field boundary
    //    kernel (it writes only ghost velocities, which nothing before the
    //    MAC correction reads, and the gas pressure);
    //  - the FEM guess, at the time the MAC correction will set (tadd = dt/2),
    //    and the two viscous guesses, for the same time (the viscous solves
    //    run after the correction; nothing before them reads their iterates).
    // The main stream joins before the MAC correction, which advances the
    // clock, so the guesses have read it by then.
    // The MAC guess runs on a third stream from the start of the step: it
    // extrapolates to the time the gas layer sets (the step's starting
    // clock, copied aside first because the gas layer advances it, plus
    // dt/2: the same sum the gas layer forms), and the main stream joins it
    // before the MAC solve.
    VDI_CUDA(cudaMemcpyAsync(S->d_time_start, S->d_time, sizeof(double), cudaMemcpyDeviceToDevice, s));
    VDI_CUDA(cudaEventRecord(S->ev_fork, s));
    VDI_CUDA(cudaStreamWaitEvent(S->s_gas, S->ev_fork, 0));
    VDI_CUDA(cudaStreamWaitEvent(S->s_guess, S->ev_fork, 0));
    VDI_TRY(guess(S, S->s_guess, SOLVER_MAC, S->q, S->q_prev, S->q_prev2, mn, 0.5 * dt, S->d_time_start));
    VDI_CUDA(cudaEventRecord(S->ev_guess, S->s_guess));
    // tracers first (fluid_2d.cc:98), before anything rewrites u, v or
    // their ghost cells
    VDI_TRY(launch_tracers(s, g, S->f, S->d_tm, S->prm.ntrace, dt));
    VDI_TRY(launch_gas_update(S->s_gas, S->gp, S->gas, S->f.u, S->f.v, m + 4, S->d_vframe, dt, S->d_time,
                              S->gas_work, S->d_err, S->d_gstats));
    // h is final for this step once the gas layer has updated it
    if (S->lcfg.mode != VDI_LIFTOFF_OFF)
        VDI_TRY(liftoff_launch(S->s_gas, S->gas.h, S->lcfg, S->d_lift, S->d_lhist, S->lcap, dt));
    VDI_CUDA(cudaEventRecord(S->ev_gas, S->s_gas));
    if (S->fused_advect) {
        // stages 1-5 in one kernel, concurrent with the gas layer; the
        // source's bottom-row term follows once the gas layer has finished
        VDI_TRY(launch_advect(s, g, S->f, dt, S->src_mac));
        VDI_CUDA(cudaEventRecord(S->ev_adv, s));
        VDI_CUDA(cudaStreamWaitEvent(s, S->ev_gas, 0));
        VDI_TRY(launch_mac_src_bottom(s, g, S->gas, dt, S->src_mac));
    } else {
        VDI_TRY(launch_stage1(s, g, S->f, dt));
        VDI_TRY(launch_stage2(s, g, S->f));
        VDI_TRY(launch_stage34(s, g, S->f, dt));
        VDI_CUDA(cudaStreamWaitEvent(s, S->ev_gas, 0));
        VDI_TRY(launch_stage5_src(s, g, S->f, S->gas, dt, S->src_mac));
        VDI_CUDA(cudaEventRecord(S->ev_adv, s));
    }
    VDI_CUDA(cudaStreamWaitEvent(S->s_gas, S->ev_adv, 0));
    VDI_TRY(launch_inviscid_bc(S->s_gas, g, S->f, S->gas, dt));
    VDI_TRY(guess(S, S->s_gas, SOLVER_FEM, S->zf, S->zf_prev, S->zf_prev2, nf, 0.5 * dt));
    const bool vside = g.implicit_visc && S->visc_guess_side;
    if (vside) {
        VDI_TRY(guess(S, S->s_gas, SOLVER_VX, S->zu, S->zu_prev, S->zu_prev2, mn, 0.5 * dt));
        VDI_TRY(guess(S, S->s_gas, SOLVER_VY, S->zv, S->zv_prev, S->zv_prev2, mn, 0.5 * dt));
    }
    VDI_CUDA(cudaEventRecord(S->ev_side, S->s_gas));
    VDI_CUDA(cudaStreamWaitEvent(s, S->ev_guess, 0));
    if (S->prm.mg_guess == VDI_GUESS_LEARNED) {
        // the network corrects the extrapolated guess from its residual
        if (!S->unet) {
            set_error("VDI_GUESS_LEARNED needs a network (vdi_sim_attach_unet)");
            return VDI_ERR_NOT_READY;
        }
        VDI_TRY(mg_residual_async(S->mg[SOLVER_MAC], s, S->src_mac, S->q, S->unet_r, S->unet_norm));
        VDI_TRY(unet_correct(S->unet, s, S->unet_r, S->unet_norm, S->q, m, n, S->unet_factor, S->unet_scale,
                             S->unet_in, S->unet_out));
    }
    VDI_TRY(mg_solve_device(S->mg[SOLVER_MAC], s, S->src_mac, S->q, prec));
    VDI_CUDA(cudaStreamWaitEvent(s, S->ev_side, 0));
    VDI_TRY(launch_mac_advect(s, g, S->f, S->gas, S->q, dt, S->d_time));
    VDI_TRY(launch_viscous_bc(s, g, S->f, S->gas));
    CellView c0v, c1v;
    if (g.implicit_visc) {
        VDI_TRY(launch_visc_rhs(s, g, S->f, S->gas, S->vfx_cur, S->vfy_cur, S->su, S->sv));
        cudaStreamCaptureStatus cs;
        VDI_CUDA(cudaStreamIsCapturing(s, &cs));
        bool par = cs == cudaStreamCaptureStatusActive;
        cudaStream_t sv = par ? S->s_vy : s;
        if (par) {
            VDI_CUDA(cudaEventRecord(S->ev_vy, s));
            VDI_CUDA(cudaStreamWaitEvent(S->s_vy, S->ev_vy, 0));
        }
        if (!vside) VDI_TRY(guess(S, s, SOLVER_VX, S->zu, S->zu_prev, S->zu_prev2, mn));
        VDI_TRY(mg_solve_device(S->mg[SOLVER_VX], s, S->su, S->zu, prec));
        if (!vside) VDI_TRY(guess(S, sv, SOLVER_VY, S->zv, S->zv_prev, S->zv_prev2, mn));
        VDI_TRY(mg_solve_device(S->mg[SOLVER_VY], sv, S->sv, S->zv, prec));
        if (par) {
            VDI_CUDA(cudaEventRecord(S->ev_vy_done, S->s_vy));
            VDI_CUDA(cudaStreamWaitEvent(s, S->ev_vy_done, 0));
        }
        c0v = CellView{S->zu, m, 0};
        c1v = CellView{S->zv, m, 0};
    } else {
        c0v = CellView{S->f.fc0, m + 4, 2 * (m + 4) + 2};
        c1v = CellView{S->f.fc1, m + 4, 2 * (m + 4) + 2};
    }
    VDI_TRY(launch_fem_rhs(s, g, S->f, S->gas, c0v, c1v, dt, S->fem_acc_edge, S->fem_acc_mid, S->src_fem));
    VDI_TRY(mg_solve_device(S->mg[SOLVER_FEM], s, S->src_fem, S->zf, prec));
    VDI_TRY(launch_vel_update(s, g, S->f, c0v, c1v, S->zf, dt));
    VDI_TRY(launch_viscous_bc(s, g, S->f, S->gas));
    // the non-inertial frame last (fluid_2d.cc:404)
    if (S->prm.nif_mode != 0)
        VDI_TRY(launch_frame(s, g, S->f, S->prm.nif_mode, S->prm.nif_a, S->prm.nif_b, S->d_vacc, S->d_vframe));
    return VDI_OK;
}

int check_errors(vdi_sim* S) {
    // one word: the step's kernels and every solve (mg_set_error_word) OR
    // their failure bits into it
    int err = 0;
    VDI_CUDA(cudaMemcpyAsync(&err, S->d_err, sizeof(int), cudaMemcpyDeviceToHost, S->s));
    VDI_CUDA(cudaStreamSynchronize(S->s));
    if (err & DEV_NONFINITE) {
        set_error("non-finite value in a residual");
        return VDI_ERR_NONFINITE;
    }
    if (err & DEV_MG_NOT_CONVERGED) {
        set_error("a multigrid solve reached its V-cycle cap");
        return VDI_ERR_MG_NOT_CONVERGED;
    }
    if (err & DEV_NEWTON) {
        set_error("gas layer: too many Newton steps");
        return VDI_ERR_NEWTON_NOT_CONVERGED;
    }
    if (err & DEV_TRI_SINGULAR) {
        set_error("gas layer: singular tridiagonal system");
        return VDI_ERR_TRI_SINGULAR;
    }
    return VDI_OK;
}

void destroy_graph(vdi_sim* S) {
    if (S->gexec) cudaGraphExecDestroy(S->gexec);
    if (S->graph) cudaGraphDestroy(S->graph);
    S->gexec = nullptr;
    S->graph = nullptr;
}

int capture_step(vdi_sim* S, double dt) {
    destroy_graph(S);
    VDI_TRY(update_visc(S, dt));
    VDI_CUDA(cudaStreamBeginCapture(S->s, cudaStreamCaptureModeRelaxed));
    int st = enqueue_step(S, dt);
    cudaGraph_t gph = nullptr;
    cudaError_t e = cudaStreamEndCapture(S->s, &gph);
    if (st != VDI_OK) {
        if (gph) cudaGraphDestroy(gph);
        return st;
    }
    VDI_CUDA(e);
    S->graph = gph;
    VDI_CUDA(cudaGraphInstantiate(&S->gexec, gph, 0));
    S->graph_dt = dt;
    return VDI_OK;
}

/** fileinfo.cc:179-191: the columns whose centres lie within nif_r of the
 * axis (from the axis when x_sym), for nif_range. */
int nif_window(vdi_params* P, double nif_r) {
    const int m = P->m;
    const double xsp = 1. / ((P->bx - P->ax) / m);
    int b = int((nif_r - P->ax) * xsp + 0.5), a;
    if (b >= m) b = m - 1;
    if (P->x_sym) a = 0;
    else {
        a = int((-nif_r - P->ax) * xsp + 0.5);
        if (a < 0) a = 0;
    }
    if (b - a <= 0) {
        set_error("Velocity window for non-inertial frame is too small");
        return VDI_ERR_CONFIG;
    }
    P->nif_a = a;
    P->nif_b = b;
    return VDI_OK;
}

int parse_cfg(const char* text, vdi_params* P) {
    // fileinfo.cc:11-193 for the gas_layer_model path
    int m = -1, n = -1, nframes = -1, glo = 0;
    double L_nd = -1, h0_nd = -1, t_end_nd = -1, tmult = -1, nul = -1, rho = -1, R = -1, V = -1, alpha = -1,
           sigma = -1, mug = -1, Pamb = -1;
    int x_sym = 0, implicit_visc = 0, ntrace = 0, nif_mode = 0;
    double nif_r = 0;
    std::istringstream in(text);
    std::string line;
    int ln = 0;
    while (std::getline(in, line)) {
        ln++;
        size_t h = line.find('#');
        if (h != std::string::npos) line = line.substr(0, h);
        std::istringstream ls(line);
        std::string key;
        if (!(ls >> key)) continue;
        std::vector<std::string> vals;
        std::string t;
        while (ls >> t) vals.push_back(t);
        auto num = [&](size_t k) -> double {
            if (k >= vals.size()) return std::nan("");
            return atof(vals[k].c_str());
        };
        if (key == "grid_points") {
            if (vals.size() != 2) { set_error("grid_points needs two values (line %d)", ln); return VDI_ERR_CONFIG; }
            m = atoi(vals[0].c_str()); n = atoi(vals[1].c_str());
        } else if (key == "L_nd") L_nd = num(0);
        else if (key == "h0_nd") h0_nd = num(0);
        else if (key == "t_end_nd") t_end_nd = num(0);
        else if (key == "frames") nframes = int(num(0));
        else if (key == "tmult") tmult = num(0);
        else if (key == "nul") nul = num(0);
        else if (key == "nul_cSt") nul = 1e-6 * num(0);
        else if (key == "rhol") rho = num(0);
        else if (key == "R") R = num(0);
        else if (key == "V") V = num(0);
        else if (key == "gamma") alpha = 1. / num(0);
        else if (key == "alpha") alpha = num(0);
        else if (key == "sigma") sigma = num(0);
        else if (key == "mug") mug = num(0);
        else if (key == "Pamb") Pamb = num(0);
        else if (key == "x_sym") x_sym = 1;
        else if (key == "implicit_visc") implicit_visc = 1;
        else if (key == "gas_layer_model") glo = 2;
        else if (key == "tracers") ntrace = atoi(vals.empty() ? "-1" : vals[0].c_str());
        else if (key == "nif_center") nif_mode = 1;                 // fileinfo.cc:96-98
        else if (key == "nif_range") {                              // fileinfo.cc:99-101
            nif_mode = 2;
            nif_r = num(0);
        } else if (key == "mr_time_output" || key == "restart_freq" || key == "output") {
        } else if (key == "gas_layer_data") {
            set_error("option '%s' is outside the GPU path (line %d)", key.c_str(), ln);
            return VDI_ERR_CONFIG;
        } else {
            set_error("Keyword '%s' not understood on line %d", key.c_str(), ln);
            return VDI_ERR_CONFIG;
        }
    }
    if (m <= 0 || n <= 0) { set_error("Grid dimensions not set"); return VDI_ERR_CONFIG; }
    const char* names[] = {"L_nd", "h0_nd", "t_end_nd", "tmult", "frames", "nul", "rhol",
                           "alpha", "mug", "Pamb", "R", "V", "sigma"};
    double vals[] = {L_nd, h0_nd, t_end_nd, tmult, double(nframes), nul, rho, alpha, mug, Pamb, R, V, sigma};
    for (int k = 0; k < 13; k++)
        if (!(vals[k] >= 0)) { set_error("Value of %s either invalid or not set", names[k]); return VDI_ERR_CONFIG; }
    if (glo != 2) { set_error("gas_layer_model must be set"); return VDI_ERR_CONFIG; }
    memset(P, 0, sizeof(*P));
    P->m = m; P->n = n; P->x_sym = x_sym; P->implicit_visc = implicit_visc;
    P->rho = rho;
    P->mu = nul * rho;                                  // fileinfo.cc:143
    double st = mug / (rho * V * R), st3 = pow(st, 1. / 3.), st23 = st3 * st3;
    double L = L_nd * R * st3;
    P->h0 = h0_nd * R * st23;
    P->t_end = t_end_nd * R * st23 / V;
    P->bx = L; P->by = L * n / m; P->ay = 0;
    if (x_sym) P->ax = 0;
    else { P->ax = -L; P->by *= 2; }
    P->tmult = tmult; P->nframes = nframes;
    P->alpha = alpha; P->mug = mug; P->Pamb = Pamb; P->R = R; P->V = V; P->sigma = sigma;
    P->mg_rtol = 1e-10;
    P->mg_max_vcycles = 200;
    P->mg_precision = VDI_MG_FP64;
    P->mg_guess = VDI_GUESS_EXTRAPOLATE;
    if (ntrace < 0) { set_error("Value of tracers invalid"); return VDI_ERR_CONFIG; }
    P->ntrace = ntrace;
    P->nif_mode = nif_mode;
    if (nif_mode == 2) VDI_TRY(nif_window(P, nif_r));
    return VDI_OK;
}

int parse_run_options(const char* text, vdi_run_options* O) {
    // fileinfo.cc:56-122: the keywords that control the run and its output
    memset(O, 0, sizeof(*O));
    std::istringstream in(text);
    std::string line;
    int ln = 0;
    while (std::getline(in, line)) {
        ln++;
        size_t h = line.find('#');
        if (h != std::string::npos) line = line.substr(0, h);
        std::istringstream ls(line);
        std::string key, t;
        if (!(ls >> key)) continue;
        std::vector<std::string> vals;
        while (ls >> t) vals.push_back(t);
        if (key == "restart_freq" || key == "tracers") {
            if (vals.size() != 1) {
                set_error("%s needs one value (line %d)", key.c_str(), ln);
                return VDI_ERR_CONFIG;
            }
            (key == "tracers" ? O->ntrace : O->restart_freq) = atoi(vals[0].c_str());
        } else if (key == "mr_time_output") {
            O->mr_time_output = 1;
        } else if (key == "output") {
            static const char* names[] = {"u", "v", "p", "pb", "pbfull", "w", "h", "fbd", "pg", "hfull",
                                          "fbdfull", "pgfull"};
            O->fflags = 0;
            for (auto& v : vals) {
                int k = 0;
                while (k < 12 && v != names[k]) k++;
                if (k == 12) {
                    set_error("Output type not understood (line %d)", ln);
                    return VDI_ERR_CONFIG;
                }
                O->fflags |= 1u << k;
            }
        } else if (key == "gas_layer_data") {
            set_error("option '%s' is outside the GPU path (line %d)", key.c_str(), ln);
            return VDI_ERR_CONFIG;
        }
    }
    if (O->restart_freq < 0 || O->ntrace < 0) {
        set_error("Value of restart_freq or tracers invalid");
        return VDI_ERR_CONFIG;
    }
    return VDI_OK;
}

}  // namespace

extern "C" {

int vdi_run_options_from_cfg(const char* text, vdi_run_options* out) {
    if (!text || !out) return VDI_ERR_INVALID_ARGUMENT;
    vdi_params P;
    int st = parse_cfg(text, &P);
    if (st != VDI_OK) return st;
    return parse_run_options(text, out);
}

const char* vdi_status_string(int s) {
    switch (s) {
        case VDI_OK: return "ok";
        case VDI_ERR_INVALID_ARGUMENT: return "invalid argument";
        case VDI_ERR_UNSUPPORTED_SIZE: return "unsupported grid size";
        case VDI_ERR_CUDA: return "CUDA error";
        case VDI_ERR_OUT_OF_MEMORY: return "out of device memory";
        case VDI_ERR_MG_NOT_CONVERGED: return "multigrid did not converge";
        case VDI_ERR_NEWTON_NOT_CONVERGED: return "Newton iteration did not converge";
        case VDI_ERR_TRI_SINGULAR: return "singular tridiagonal system";
        case VDI_ERR_NONFINITE: return "non-finite value";
        case VDI_ERR_CONFIG: return "configuration error";
        case VDI_ERR_NOT_READY: return "not ready";
    }
    return "unknown status";
}

int vdi_abi_version(void) { return VDI_ABI_VERSION; }
const char* vdi_last_error(void) { return g_err; }

int vdi_params_from_cfg(const char* cfg_text, vdi_params* out) {
    if (!cfg_text || !out) return VDI_ERR_INVALID_ARGUMENT;
    return parse_cfg(cfg_text, out);
}

int vdi_sim_create(const vdi_params* prm, void* stream, vdi_sim** out) {
    if (!prm || !out || prm->m < 4 || prm->n < 4) {
        set_error("vdi_sim_create: invalid parameters");
        return VDI_ERR_INVALID_ARGUMENT;
    }
    if (prm->ntrace < 0 || prm->nif_mode < 0 || prm->nif_mode > 2 ||
        (prm->nif_mode == 2 && !(prm->nif_a >= 0 && prm->nif_a < prm->nif_b && prm->nif_b <= prm->m))) {
        set_error("vdi_sim_create: invalid tracer or non-inertial frame parameters");
        return VDI_ERR_INVALID_ARGUMENT;
    }
    vdi_sim* S = new vdi_sim();
    S->prm = *prm;
    if (S->prm.mg_rtol <= 0) S->prm.mg_rtol = 1e-10;
    if (S->prm.mg_max_vcycles <= 0) S->prm.mg_max_vcycles = 200;
    Grid& g = S->g;
    const vdi_params& P = S->prm;
    g.m = P.m; g.n = P.n; g.x_sym = P.x_sym; g.implicit_visc = P.implicit_visc;
    g.blk_x = 32; g.blk_y = 8;
    if (const char* e = getenv("VDI_FUSED_ADVECT")) S->fused_advect = atoi(e) != 0;
    if (const char* e = getenv("VDI_VISC_GUESS_SIDE")) S->visc_guess_side = atoi(e) != 0;
    g.ax = P.ax; g.ay = P.ay; g.bx = P.bx; g.by = P.by;
    // fluid_2d.cc:15-17
    g.dx = (P.bx - P.ax) / P.m;
    g.dy = (P.by - P.ay) / P.n;
    g.xsp = 1. / g.dx; g.ysp = 1. / g.dy;
    g.xxsp = g.xsp * g.xsp; g.yysp = g.ysp * g.ysp;
    g.rho = P.rho; g.rhoinv = 1. / P.rho; g.mu = P.mu; g.muinv = 1. / P.mu;
    g.viscfac = P.implicit_visc ? g.rhoinv * g.mu * 0.5 : g.rhoinv * g.mu;   // fluid_2d.cc:164
    S->dt_reg = P.implicit_visc ? g.dx * P.tmult : g.dx * g.dx * P.rho * g.muinv * P.tmult * 0.25;
    GasPrm& gp = S->gp;
    gp.m = P.m; gp.x_sym = P.x_sym; gp.ax = P.ax;
    gp.dx = (P.bx - P.ax) / P.m;       // gas_layer.cc:9
    gp.xsp = 1. / gp.dx; gp.xxsp = gp.xsp * gp.xsp;
    gp.alpha = P.alpha; gp.mu = P.mug; gp.Pamb = P.Pamb; gp.R = P.R; gp.sigma = P.sigma;

    auto fail = [&](int st) {
        vdi_sim_destroy(S);
        return st;
    };
    int st;
    if (stream) {
        S->s = static_cast<cudaStream_t>(stream);
    } else {
        if (cudaStreamCreateWithFlags(&S->s, cudaStreamNonBlocking) != cudaSuccess) return fail(VDI_ERR_CUDA);
        S->own_stream = true;
    }
    if (cudaStreamCreateWithFlags(&S->s_gas, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&S->s_vy, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&S->s_guess, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->ev_guess, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->ev_gas, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->ev_vy, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->ev_vy_done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->ev_adv, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&S->ev_side, cudaEventDisableTiming) != cudaSuccess)
        return fail(VDI_ERR_CUDA);
    size_t NG = ghosted(S);
    double** fptrs[] = {&S->f.u, &S->f.v, &S->f.p, &S->f.ux, &S->f.uy, &S->f.vx, &S->f.vy,
                        &S->f.ud, &S->f.vd, &S->f.ul, &S->f.vl, &S->f.ur, &S->f.vr, &S->f.uu, &S->f.vu,
                        &S->f.ud2, &S->f.vd2, &S->f.ul2, &S->f.vl2, &S->f.ur2, &S->f.vr2, &S->f.uu2, &S->f.vu2,
                        &S->f.fc0, &S->f.fc1};
    for (auto pp : fptrs)
        if ((st = alloc_zero(S, pp, NG)) != VDI_OK) return fail(st);
    const int m = P.m, n = P.n;
    size_t mn = size_t(m) * n, nf = size_t(m + 1) * (n + 1);
    double** gptrs[] = {&S->gas.gp, &S->gas.gp_old, &S->gas.pg, &S->gas.pg_old, &S->gas.hx};
    for (auto pp : gptrs)
        if ((st = alloc_zero(S, pp, m + 1)) != VDI_OK) return fail(st);
    double** gptrs2[] = {&S->gas.tau, &S->gas.tau_old};
    for (auto pp : gptrs2)
        if ((st = alloc_zero(S, pp, m + 4)) != VDI_OK) return fail(st);
    double** gptrs3[] = {&S->gas.h, &S->gas.ht, &S->gas.fbd};
    for (auto pp : gptrs3)
        if ((st = alloc_zero(S, pp, m)) != VDI_OK) return fail(st);
    if ((st = alloc_zero(S, &S->gas_work, gas_work_doubles(m))) != VDI_OK) return fail(st);
    double** cells[] = {&S->src_mac, &S->q,  &S->q_prev,  &S->su,      &S->sv,      &S->zu,
                        &S->zu_prev, &S->zv, &S->zv_prev, &S->q_prev2, &S->zu_prev2, &S->zv_prev2};
    for (auto pp : cells)
        if ((st = alloc_zero(S, pp, mn)) != VDI_OK) return fail(st);
    double** nodes[] = {&S->src_fem, &S->zf, &S->zf_prev, &S->zf_prev2};
    for (auto pp : nodes)
        if ((st = alloc_zero(S, pp, nf)) != VDI_OK) return fail(st);
    double* misc;
    if ((st = alloc_zero(S, &misc, 2 + 4 * (sizeof(GuessHist) / 8 + 1))) != VDI_OK) return fail(st);
    S->d_time = misc;
    S->d_vframe = misc + 1;
    S->hist = reinterpret_cast<GuessHist*>(misc + 2);
    if (P.ntrace > 0 && (st = alloc_zero(S, &S->d_tm, 2 * size_t(P.ntrace))) != VDI_OK) return fail(st);
    if ((st = alloc_zero(S, &S->d_vacc, 1)) != VDI_OK) return fail(st);
    if ((st = alloc_zero(S, &S->d_time_aside, 1)) != VDI_OK) return fail(st);
    if ((st = alloc_zero(S, &S->d_time_start, 1)) != VDI_OK) return fail(st);
    double* ebuf;
    if ((st = alloc_zero(S, &ebuf, 1 + sizeof(GasStats) / 8 + 1)) != VDI_OK) return fail(st);
    S->d_err = reinterpret_cast<int*>(ebuf);
    S->d_gstats = reinterpret_cast<GasStats*>(ebuf + 1);
    // the four linear systems (fluid_2d.cc:19-21)
    if ((st = mg_create(VDI_MG_MAC, m, n, g.xxsp, g.yysp, P.x_sym, &S->mg[SOLVER_MAC])) != VDI_OK) return fail(st);
    if ((st = mg_create(VDI_MG_FEM, m + 1, n + 1, g.dx, g.dy, P.x_sym, &S->mg[SOLVER_FEM])) != VDI_OK)
        return fail(st);
    if (P.implicit_visc) {
        if ((st = mg_create(VDI_MG_VISC_U, m, n, 1., 1., P.x_sym, &S->mg[SOLVER_VX])) != VDI_OK) return fail(st);
        if ((st = mg_create(VDI_MG_VISC_V, m, n, 1., 1., P.x_sym, &S->mg[SOLVER_VY])) != VDI_OK) return fail(st);
    }
    for (int k = 0; k < 4; k++)
        if (S->mg[k] && ((st = mg_configure(S->mg[k], S->prm.mg_rtol, S->prm.mg_max_vcycles)) != VDI_OK ||
                         (st = mg_set_error_word(S->mg[k], S->d_err)) != VDI_OK))
            return fail(st);
    double* lbuf;
    if ((st = alloc_zero(S, &lbuf, sizeof(LiftoffState) / 8 + 1)) != VDI_OK) return fail(st);
    S->d_lift = reinterpret_cast<LiftoffState*>(lbuf);
    if (P.m <= LIFTOFF_MAX_M &&
        liftoff_config(P.m, P.ax, gp.dx, VDI_LIFTOFF_SMOOTHED, 1, P.R, P.V, &S->lcfg) != VDI_OK)
        S->lcfg.mode = VDI_LIFTOFF_OFF;
    // mgs_fem::a_cc on the bottom row (mgs_fem.hh:55-57)
    double dydx = g.dy / g.dx, dxdy = g.dx / g.dy, fm = 4. / 3. * (dxdy + dydx);
    S->fem_acc_edge = 0.5 * 0.5 * fm;
    S->fem_acc_mid = 1. * 0.5 * fm;
    *out = S;
    return VDI_OK;
}

int vdi_sim_attach_unet(vdi_sim* S, vdi_unet* net, int factor, double out_scale) {
    if (!S || !net || (factor != 1 && factor != 2 && factor != 4 && factor != 8)) return VDI_ERR_INVALID_ARGUMENT;
    int H, W;
    unet_dims(net, &H, &W);
    if (S->prm.m / factor != W || S->prm.n / factor != H || S->prm.m % factor || S->prm.n % factor) {
        set_error("vdi_sim_attach_unet: the network grid %dx%d does not match %dx%d / %d", W, H, S->prm.m,
                  S->prm.n, factor);
        return VDI_ERR_INVALID_ARGUMENT;
    }
    if (!S->unet_r) {
        int st;
        if ((st = alloc_zero(S, &S->unet_r, size_t(S->prm.m) * S->prm.n)) != VDI_OK) return st;
        if ((st = alloc_zero(S, &S->unet_norm, 1)) != VDI_OK) return st;
        double* f;
        if ((st = alloc_zero(S, &f, size_t(H) * W)) != VDI_OK) return st;   // 2 float arrays
        S->unet_in = reinterpret_cast<float*>(f);
        S->unet_out = S->unet_in + size_t(H) * W;
    }
    S->unet = net;
    S->unet_factor = factor;
    // scale of the output: out_scale * rms(r) / xxsp
    S->unet_scale = out_scale / S->g.xxsp;
    destroy_graph(S);
    // one eager correction on zeros sets the kernels' shared-memory limits
    // before any stream capture
    VDI_CUDA(cudaMemsetAsync(S->unet_r, 0, sizeof(double) * S->prm.m * S->prm.n, S->s));
    VDI_CUDA(cudaMemsetAsync(S->unet_norm, 0, sizeof(double), S->s));
    VDI_TRY(unet_correct(net, S->s, S->unet_r, S->unet_norm, S->unet_r, S->prm.m, S->prm.n, factor, 0.,
                         S->unet_in, S->unet_out));
    VDI_CUDA(cudaStreamSynchronize(S->s));
    return VDI_OK;
}

int vdi_sim_destroy(vdi_sim* S) {
    if (!S) return VDI_OK;
    if (S->s) cudaStreamSynchronize(S->s);
    destroy_graph(S);
    for (int k = 0; k < 4; k++)
        if (S->mg[k]) mg_destroy(S->mg[k]);
    for (auto p : S->bufs) cudaFree(p);
    if (S->ev_fork) cudaEventDestroy(S->ev_fork);
    if (S->ev_gas) cudaEventDestroy(S->ev_gas);
    if (S->ev_vy) cudaEventDestroy(S->ev_vy);
    if (S->ev_vy_done) cudaEventDestroy(S->ev_vy_done);
    if (S->ev_adv) cudaEventDestroy(S->ev_adv);
    if (S->ev_side) cudaEventDestroy(S->ev_side);
    if (S->ev_guess) cudaEventDestroy(S->ev_guess);
    if (S->s_gas) cudaStreamDestroy(S->s_gas);
    if (S->s_vy) cudaStreamDestroy(S->s_vy);
    if (S->s_guess) cudaStreamDestroy(S->s_guess);
    if (S->own_stream && S->s) cudaStreamDestroy(S->s);
    delete S;
    return VDI_OK;
}

/** fluid_2d::init_tracers (fluid_2d.cc:495-502): positions from the
 * process's rand(), uniform over the domain. */
static int place_tracers(vdi_sim* S) {
    const vdi_params& P = S->prm;
    std::vector<double> tm(2 * size_t(P.ntrace));
    for (size_t k = 0; k < tm.size(); k += 2) {
        tm[k] = P.ax + (P.bx - P.ax) / RAND_MAX * static_cast<double>(rand());
        tm[k + 1] = P.ay + (P.by - P.ay) / RAND_MAX * static_cast<double>(rand());
    }
    VDI_CUDA(cudaMemcpyAsync(S->d_tm, tm.data(), tm.size() * sizeof(double), cudaMemcpyHostToDevice, S->s));
    VDI_CUDA(cudaStreamSynchronize(S->s));
    return VDI_OK;
}

/** Restarts the lift-off search with the current state as state 0. */
static int liftoff_restart(vdi_sim* S) {
    VDI_TRY(liftoff_reset_async(S->s, S->d_lift));
    if (S->lcfg.mode != VDI_LIFTOFF_OFF)
        VDI_TRY(liftoff_launch(S->s, S->gas.h, S->lcfg, S->d_lift, S->d_lhist, S->lcap, 0.));
    return VDI_OK;
}

static int reset_histories(vdi_sim* S) {
    cudaStream_t s = S->s;
    size_t mn = size_t(S->prm.m) * S->prm.n, nf = size_t(S->prm.m + 1) * (S->prm.n + 1);
    VDI_CUDA(cudaMemsetAsync(S->hist, 0, 4 * sizeof(GuessHist), s));
    double* zs[] = {S->q, S->q_prev, S->zu, S->zu_prev, S->zv, S->zv_prev, S->q_prev2, S->zu_prev2, S->zv_prev2};
    for (auto z : zs) VDI_CUDA(cudaMemsetAsync(z, 0, mn * sizeof(double), s));
    VDI_CUDA(cudaMemsetAsync(S->zf, 0, nf * sizeof(double), s));
    VDI_CUDA(cudaMemsetAsync(S->zf_prev, 0, nf * sizeof(double), s));
    VDI_CUDA(cudaMemsetAsync(S->zf_prev2, 0, nf * sizeof(double), s));
    return VDI_OK;
}

int vdi_sim_init_fields(vdi_sim* S) {
    if (!S) return VDI_ERR_INVALID_ARGUMENT;
    cudaStream_t s = S->s;
    size_t NG = ghosted(S);
    VDI_CUDA(cudaMemsetAsync(S->f.u, 0, NG * 8, s));
    VDI_CUDA(cudaMemsetAsync(S->f.v, 0, NG * 8, s));
    VDI_CUDA(cudaMemsetAsync(S->f.p, 0, NG * 8, s));
    VDI_CUDA(cudaMemsetAsync(S->gas.tau, 0, (S->prm.m + 4) * 8, s));
    double tv[2] = {0., S->prm.V};
    VDI_CUDA(cudaMemcpyAsync(S->d_time, tv, sizeof(tv), cudaMemcpyHostToDevice, s));
    VDI_TRY(reset_histories(S));
    VDI_TRY(launch_gas_init(s, S->gp, S->gas, S->prm.h0, S->prm.V));
    VDI_TRY(launch_inviscid_bc(s, S->g, S->f, S->gas, 0.));
    VDI_TRY(launch_viscous_bc(s, S->g, S->f, S->gas));
    VDI_TRY(liftoff_restart(S));
    if (S->prm.ntrace > 0) VDI_TRY(place_tracers(S));   // fluid_2d_sio.cc:30
    VDI_CUDA(cudaStreamSynchronize(s));
    return VDI_OK;
}

int vdi_sim_get_params(const vdi_sim* S, vdi_params* out) {
    if (!S || !out) return VDI_ERR_INVALID_ARGUMENT;
    *out = S->prm;
    return VDI_OK;
}

int vdi_sim_init_tracers(vdi_sim* S) {
    if (!S) return VDI_ERR_INVALID_ARGUMENT;
    if (S->prm.ntrace == 0) return VDI_OK;
    return place_tracers(S);
}

int vdi_sim_update_tracers(vdi_sim* S, double dt) {
    if (!S || !std::isfinite(dt)) return VDI_ERR_INVALID_ARGUMENT;
    if (S->prm.ntrace == 0) return VDI_OK;
    VDI_TRY(launch_tracers(S->s, S->g, S->f, S->d_tm, S->prm.ntrace, dt));
    VDI_CUDA(cudaStreamSynchronize(S->s));
    return VDI_OK;
}

int vdi_sim_set_nif_mode(vdi_sim* S, int mode, double w) {
    if (!S || mode < 0 || mode > 2) return VDI_ERR_INVALID_ARGUMENT;
    vdi_params P = S->prm;
    P.nif_mode = mode;
    if (mode == 2) VDI_TRY(nif_window(&P, w));
    VDI_CUDA(cudaStreamSynchronize(S->s));
    S->prm.nif_mode = P.nif_mode;
    S->prm.nif_a = P.nif_a;
    S->prm.nif_b = P.nif_b;
    destroy_graph(S);   // the captured step holds the previous mode
    return VDI_OK;
}

int vdi_gas_update(vdi_sim* S, double dt) {
    if (!S || !(dt > 0)) return VDI_ERR_INVALID_ARGUMENT;
    // the kernel advances the clock it is given by dt/2 (the step's
    // half-time); run alone, it gets a copy so the simulation's clock stays
    VDI_CUDA(cudaMemcpyAsync(S->d_time_aside, S->d_time, sizeof(double), cudaMemcpyDeviceToDevice, S->s));
    VDI_TRY(launch_gas_update(S->s, S->gp, S->gas, S->f.u, S->f.v, S->prm.m + 4, S->d_vframe, dt,
                              S->d_time_aside, S->gas_work, S->d_err, S->d_gstats));
    return check_errors(S);
}

int vdi_gas_init_fields(vdi_sim* S) {
    if (!S) return VDI_ERR_INVALID_ARGUMENT;
    VDI_CUDA(cudaMemsetAsync(S->gas.tau, 0, (S->prm.m + 4) * 8, S->s));
    VDI_TRY(launch_gas_init(S->s, S->gp, S->gas, S->prm.h0, S->prm.V));
    VDI_CUDA(cudaStreamSynchronize(S->s));
    return VDI_OK;
}

int vdi_sim_get_tracers(vdi_sim* S, double* h_xy, long count) {
    if (!S || (count > 0 && !h_xy) || count != 2L * S->prm.ntrace) return VDI_ERR_INVALID_ARGUMENT;
    if (count == 0) return VDI_OK;
    VDI_CUDA(cudaStreamSynchronize(S->s));
    VDI_CUDA(cudaMemcpy(h_xy, S->d_tm, size_t(count) * sizeof(double), cudaMemcpyDeviceToHost));
    return VDI_OK;
}

int vdi_sim_set_tracers(vdi_sim* S, const double* h_xy, long count) {
    if (!S || (count > 0 && !h_xy) || count != 2L * S->prm.ntrace) return VDI_ERR_INVALID_ARGUMENT;
    if (count == 0) return VDI_OK;
    VDI_CUDA(cudaStreamSynchronize(S->s));
    VDI_CUDA(cudaMemcpy(S->d_tm, h_xy, size_t(count) * sizeof(double), cudaMemcpyHostToDevice));
    return VDI_OK;
}

int vdi_sim_timestep_select(const vdi_sim* S, double interval, double* adt, int* nsteps) {
    if (!S || !adt) return VDI_ERR_INVALID_ARGUMENT;
    int l = static_cast<int>(interval / S->dt_reg) + 1;   // fluid_2d.hh:82-86
    *adt = interval / l;
    if (nsteps) *nsteps = l;
    return VDI_OK;
}

int vdi_sim_step_forward(vdi_sim* S, double dt, int nsteps) {
    if (!S || !(dt > 0) || nsteps < 0) return VDI_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < nsteps; k++) {
        if (S->use_graph) {
            if (!S->gexec || S->graph_dt != dt) VDI_TRY(capture_step(S, dt));
            VDI_CUDA(cudaGraphLaunch(S->gexec, S->s));
        } else {
            VDI_TRY(update_visc(S, dt));
            VDI_TRY(enqueue_step(S, dt));
        }
        S->steps++;
    }
    return check_errors(S);
}

int vdi_sim_use_graph(vdi_sim* S, int enable) {
    if (!S) return VDI_ERR_INVALID_ARGUMENT;
    S->use_graph = enable != 0;
    if (!S->use_graph) destroy_graph(S);
    return VDI_OK;
}

int vdi_sim_synchronize(vdi_sim* S) {
    if (!S) return VDI_ERR_INVALID_ARGUMENT;
    return check_errors(S);
}

int vdi_sim_get_state(vdi_sim* S, vdi_state* h) {
    if (!S || !h) return VDI_ERR_INVALID_ARGUMENT;
    VDI_CUDA(cudaStreamSynchronize(S->s));
    size_t NG = ghosted(S) * 8;
    int m = S->prm.m;
    struct {
        double* dst;
        const double* src;
        size_t bytes;
    } cp[] = {{h->u, S->f.u, NG},        {h->v, S->f.v, NG},          {h->p, S->f.p, NG},
              {h->gp, S->gas.gp, (m + 1) * 8u}, {h->tau, S->gas.tau, (m + 4) * 8u}, {h->h, S->gas.h, m * 8u},
              {h->fbd, S->gas.fbd, m * 8u}, {h->pg, S->gas.pg, (m + 1) * 8u}, {h->ht, S->gas.ht, m * 8u}};
    for (auto& c : cp)
        if (c.dst) VDI_CUDA(cudaMemcpy(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost));
    double tv[2];
    VDI_CUDA(cudaMemcpy(tv, S->d_time, sizeof(tv), cudaMemcpyDeviceToHost));
    h->time = tv[0];
    h->Vframe = tv[1];
    return VDI_OK;
}

int vdi_sim_set_state(vdi_sim* S, const vdi_state* h) {
    if (!S || !h || !h->u || !h->v || !h->p || !h->gp || !h->tau || !h->h || !h->fbd || !h->pg || !h->ht)
        return VDI_ERR_INVALID_ARGUMENT;
    VDI_CUDA(cudaStreamSynchronize(S->s));
    size_t NG = ghosted(S) * 8;
    int m = S->prm.m;
    struct {
        double* dst;
        const double* src;
        size_t bytes;
    } cp[] = {{S->f.u, h->u, NG},        {S->f.v, h->v, NG},          {S->f.p, h->p, NG},
              {S->gas.gp, h->gp, (m + 1) * 8u}, {S->gas.tau, h->tau, (m + 4) * 8u}, {S->gas.h, h->h, m * 8u},
              {S->gas.fbd, h->fbd, m * 8u}, {S->gas.pg, h->pg, (m + 1) * 8u}, {S->gas.ht, h->ht, m * 8u}};
    for (auto& c : cp) VDI_CUDA(cudaMemcpy(c.dst, c.src, c.bytes, cudaMemcpyHostToDevice));
    double tv[2] = {h->time, h->Vframe};
    VDI_CUDA(cudaMemcpy(S->d_time, tv, sizeof(tv), cudaMemcpyHostToDevice));
    // hx is derived from h, as the reference's restart loader does
    // (gas_layer_solve.cc:318); the multigrid history restarts (mgs_common.cc:22-27)
    std::vector<double> hh(h->h, h->h + m), hx(m + 1);
    for (int i = 1; i < m; i++) hx[i] = S->gp.xsp * (hh[i] - hh[i - 1]);
    hx[0] = S->prm.x_sym ? 0 : hx[1];
    hx[m] = hx[m - 1];
    VDI_CUDA(cudaMemcpy(S->gas.hx, hx.data(), (m + 1) * 8, cudaMemcpyHostToDevice));
    VDI_TRY(reset_histories(S));
    VDI_TRY(liftoff_restart(S));
    VDI_CUDA(cudaStreamSynchronize(S->s));
    return VDI_OK;
}

int vdi_sim_liftoff_setup(vdi_sim* S, int mode, int every, long history) {
    if (!S || history < 0) return VDI_ERR_INVALID_ARGUMENT;
    LiftoffCfg c{};
    if (mode != VDI_LIFTOFF_OFF)
        VDI_TRY(liftoff_config(S->prm.m, S->prm.ax, S->gp.dx, mode, every, S->prm.R, S->prm.V, &c));
    VDI_CUDA(cudaStreamSynchronize(S->s));
    destroy_graph(S);
    if (S->d_lhist) {
        for (auto& p : S->bufs)
            if (p == reinterpret_cast<double*>(S->d_lhist)) p = nullptr;
        VDI_CUDA(cudaFree(S->d_lhist));
        S->d_lhist = nullptr;
    }
    S->lcap = 0;
    if (history > 0) {
        double* hb;
        VDI_TRY(alloc_zero(S, &hb, 2 * size_t(history)));
        S->d_lhist = reinterpret_cast<double2*>(hb);
        S->lcap = history;
    }
    S->lcfg = c;
    S->lcfg.mode = mode;
    VDI_TRY(liftoff_restart(S));
    VDI_CUDA(cudaStreamSynchronize(S->s));
    return VDI_OK;
}

int vdi_sim_liftoff(vdi_sim* S, vdi_liftoff* out, double* h_xmin, double* h_fmin, long cap) {
    if (!S || !out || cap < 0 || (cap > 0 && (!h_xmin || !h_fmin))) return VDI_ERR_INVALID_ARGUMENT;
    VDI_CUDA(cudaStreamSynchronize(S->s));
    LiftoffState st;
    VDI_CUDA(cudaMemcpy(&st, S->d_lift, sizeof(st), cudaMemcpyDeviceToHost));
    memset(out, 0, sizeof(*out));
    out->states = st.count;
    out->min_state = st.gimin;
    out->min_height = st.gfmin;
    out->min_x = st.gxmin;
    out->interval = st.interval;
    out->searching = st.hsearch;
    out->ev_found = !st.efield;
    out->last_x = st.last_x;
    out->last_height = st.last_f;
    // the tool's summary line (tt_analysis.cc:169-171)
    const double gtmin = st.gimin * st.interval;
    out->t_rel = gtmin - S->prm.h0 / S->prm.V;
    out->t_rel_ev = gtmin - st.tmin0_ev;
    out->percent = st.count > 1 ? 100. * float(st.gimin) / float(st.count - 1) : 0.;
    long n = std::min(cap, std::min(st.count, S->lcap));
    if (n > 0) {
        std::vector<double2> hb(n);
        VDI_CUDA(cudaMemcpy(hb.data(), S->d_lhist, n * sizeof(double2), cudaMemcpyDeviceToHost));
        for (long k = 0; k < n; k++) {
            h_xmin[k] = hb[k].x;
            h_fmin[k] = hb[k].y;
        }
    }
    return VDI_OK;
}

int vdi_sim_stats(vdi_sim* S, vdi_stats* out, int reset) {
    if (!S || !out) return VDI_ERR_INVALID_ARGUMENT;
    VDI_CUDA(cudaStreamSynchronize(S->s));
    memset(out, 0, sizeof(*out));
    out->steps = S->steps;
    for (int k = 0; k < 4; k++) {
        if (!S->mg[k]) continue;
        SolveCtl c;
        VDI_CUDA(cudaMemcpy(&c, mg_ctl(S->mg[k]), sizeof(SolveCtl), cudaMemcpyDeviceToHost));
        out->solves[k] = long(c.solves);
        out->vcycles[k] = long(c.vcycles);
        out->last_rel_res[k] = c.last_rel;
        if (reset) {
            c.solves = 0;
            c.vcycles = 0;
            VDI_CUDA(cudaMemcpy(mg_ctl(S->mg[k]), &c, sizeof(SolveCtl), cudaMemcpyHostToDevice));
        }
    }
    // launches: per step the gas-layer update, the four stencil stages, the
    // MAC correction, two boundary kernels, the FEM source, the velocity update
    // and the final boundary kernel (+1 viscous source when implicit); per
    // solve the initial guess and the start check; per solve-loop iteration
    // the kernels of its V-cycle;
    // per step the lift-off search when it is on, the tracers and the two
    // frame kernels when those are on, and with the learned guess the
    // residual kernel and the network's correction.
    long per_step = 11 - (S->fused_advect ? 2 : 0) + (S->prm.implicit_visc ? 1 : 0) + (S->lcfg.mode != VDI_LIFTOFF_OFF ? 1 : 0) +
                    (S->prm.ntrace > 0 ? 1 : 0) + (S->prm.nif_mode != 0 ? 2 : 0) +
                    (S->prm.mg_guess == VDI_GUESS_LEARNED ? 1 + unet_kernels_per_correction() : 0);
    long launches = S->steps * per_step;
    for (int k = 0; k < 4; k++) {
        if (!S->mg[k]) continue;
        // the guess kernel and the start check
        launches += out->solves[k] * 2 +
                    out->vcycles[k] * mg_kernels_per_iteration(S->mg[k], S->prm.mg_precision);
    }
    out->kernel_launches = launches;
    GasStats gs;
    VDI_CUDA(cudaMemcpy(&gs, S->d_gstats, sizeof(gs), cudaMemcpyDeviceToHost));
    out->newton_steps = long(gs.newton_steps);
    out->tri_pivot_fallbacks = long(gs.pivot_fallbacks);
    out->height_fixed_point_iters = long(gs.fixed_point_iters);
    if (reset) {
        VDI_CUDA(cudaMemset(S->d_gstats, 0, sizeof(GasStats)));
        S->steps = 0;
    }
    return VDI_OK;
}

int vdi_sim_device_field(vdi_sim* S, int which, double** d_ptr, size_t* count) {
    if (!S || !d_ptr) return VDI_ERR_INVALID_ARGUMENT;
    int m = S->prm.m;
    switch (which) {
        case 0: *d_ptr = S->f.u; if (count) *count = ghosted(S); break;
        case 1: *d_ptr = S->f.v; if (count) *count = ghosted(S); break;
        case 2: *d_ptr = S->f.p; if (count) *count = ghosted(S); break;
        case 3: *d_ptr = S->gas.h; if (count) *count = m; break;
        case 4: *d_ptr = S->gas.pg; if (count) *count = m + 1; break;
        case 5: *d_ptr = S->gas.gp; if (count) *count = m + 1; break;
        case 6: *d_ptr = S->src_mac; if (count) *count = size_t(m) * S->prm.n; break;
        case 7: *d_ptr = S->q; if (count) *count = size_t(m) * S->prm.n; break;
        case 8: *d_ptr = S->src_fem; if (count) *count = size_t(m + 1) * (S->prm.n + 1); break;
        case 9: *d_ptr = S->gas.gp_old; if (count) *count = m + 1; break;
        case 10: *d_ptr = S->gas.tau; if (count) *count = m + 4; break;
        case 11: *d_ptr = S->gas.tau_old; if (count) *count = m + 4; break;
        case 12: *d_ptr = S->gas.ht; if (count) *count = m; break;
        case 13: *d_ptr = S->gas.fbd; if (count) *count = m; break;
        default: return VDI_ERR_INVALID_ARGUMENT;
    }
    return VDI_OK;
}

int vdi_sim_vcycle_bytes(const vdi_sim* S, int precision, double* out4) {
    if (!S || !out4) return VDI_ERR_INVALID_ARGUMENT;
    if (precision != VDI_MG_FP64 && precision != VDI_MG_MIXED && precision != VDI_MG_HYBRID)
        return VDI_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 4; k++) {
        out4[k] = 0;
        const MG* g = S->mg[k];
        if (!g) continue;
        if (precision == VDI_MG_FP64) out4[k] = mg_vcycle_bytes(g, 8, 8);
        else if (precision == VDI_MG_HYBRID) out4[k] = mg_vcycle_bytes(g, 8, 4);
        else out4[k] = mg_vcycle_bytes(g, 4, 4) + 40. * mg_fine_size(g);
    }
    return VDI_OK;
}

// ------------------------------------------------------------ multigrid
struct vdi_mg {
    MG* g = nullptr;
    cudaStream_t s = nullptr;
    // solves replayed from a captured graph, per (b, z, precision): the
    // start kernel and a conditional WHILE node over the V-cycles, so a
    // solve is one launch and one read of the control block
    struct Replay {
        const double* b;
        double* z;
        int precision;
        cudaGraphExec_t exec;
    };
    std::vector<Replay> replays;
    std::vector<std::pair<const double*, double*>> seen;   // solved once eagerly
    cudaStream_t cap = nullptr;                             // capture stream
    double rtol = -1;
    int max_it = -1;
};

namespace {

bool solve_graphs_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("VDI_MG_SOLVE_GRAPH");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

/** The solve of vdi_mg_solve from a captured graph (the second and later
 * solves of the same arrays). */
int mg_solve_replay(vdi_mg* h, const double* b, double* z, double rtol, int max_it, int precision, int* vcycles,
                    double* rel_res) {
    if (rtol != h->rtol || max_it != h->max_it) {
        VDI_TRY(mg_configure(h->g, rtol, max_it));
        h->rtol = rtol;
        h->max_it = max_it;
    }
    cudaGraphExec_t exec = nullptr;
    for (auto& r : h->replays)
        if (r.b == b && r.z == z && r.precision == precision) exec = r.exec;
    if (!exec) {
        if (!h->cap) VDI_CUDA(cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking));
        VDI_CUDA(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
        int st = mg_record_graph_solve(h->g, h->cap, b, z, precision);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(h->cap, &graph);
        if (st != VDI_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        VDI_CUDA(e);
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        VDI_CUDA(e);
        h->replays.push_back(vdi_mg::Replay{b, z, precision, exec});
    }
    VDI_CUDA(cudaGraphLaunch(exec, h->s));
    SolveCtl c;
    VDI_CUDA(cudaMemcpyAsync(&c, mg_ctl(h->g), sizeof(SolveCtl), cudaMemcpyDeviceToHost, h->s));
    VDI_CUDA(cudaStreamSynchronize(h->s));
    if (vcycles) *vcycles = c.it;
    if (rel_res) *rel_res = c.bnorm2 > 0 ? std::sqrt(c.rnorm2 / c.bnorm2) : 0.;
    if (c.status & DEV_NONFINITE) {
        set_error("multigrid: non-finite residual");
        return VDI_ERR_NONFINITE;
    }
    if (c.status & DEV_MG_NOT_CONVERGED) {
        set_error("multigrid: %d V-cycles without reaching rtol %.3g (rel. residual %.3g)", c.it, rtol,
                  c.bnorm2 > 0 ? std::sqrt(c.rnorm2 / c.bnorm2) : 0.);
        return VDI_ERR_MG_NOT_CONVERGED;
    }
    return VDI_OK;
}

}  // namespace

int vdi_mg_create(int kind, int m, int n, double c1, double c2, int x_sym, void* stream, vdi_mg** out) {
    if (!out) return VDI_ERR_INVALID_ARGUMENT;
    vdi_mg* h = new vdi_mg();
    h->s = static_cast<cudaStream_t>(stream);
    double a = c1, b = c2;
    if (kind == VDI_MG_MAC || kind == VDI_MG_MAC_NEUMANN) {
        // mgs_mac.cc:23-27 (test constructor): xxsp = 1/(dx*dx)
        a = 1. / (c1 * c1);
        b = 1. / (c2 * c2);
    }
    int st = mg_create(kind, m, n, a, b, x_sym, &h->g);
    if (st != VDI_OK) {
        delete h;
        return st;
    }
    *out = h;
    return VDI_OK;
}

int vdi_mg_destroy(vdi_mg* h) {
    if (!h) return VDI_OK;
    for (auto& r : h->replays) cudaGraphExecDestroy(r.exec);
    if (h->cap) cudaStreamDestroy(h->cap);
    if (h->g) mg_destroy(h->g);
    delete h;
    return VDI_OK;
}

int vdi_mg_setup(vdi_mg* h) { return h ? VDI_OK : VDI_ERR_INVALID_ARGUMENT; }

int vdi_mg_solve(vdi_mg* h, const double* d_b, double* d_z, double rtol, int max_vcycles, int precision,
                 vdi_mg_result* res) {
    if (!h || !d_b || !d_z || !(rtol > 0) || max_vcycles < 0) return VDI_ERR_INVALID_ARGUMENT;
    int v = 0;
    double r = 0;
    int st;
    const std::pair<const double*, double*> key{d_b, d_z};
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (h->s) VDI_CUDA(cudaStreamIsCapturing(h->s, &cs));
    const bool again = std::find(h->seen.begin(), h->seen.end(), key) != h->seen.end();
    if (solve_graphs_enabled() && again && cs == cudaStreamCaptureStatusNone) {
        st = mg_solve_replay(h, d_b, d_z, rtol, max_vcycles, precision, &v, &r);
    } else {
        st = mg_solve(h->g, h->s, d_b, d_z, rtol, max_vcycles, precision, &v, &r);
        h->rtol = rtol;
        h->max_it = max_vcycles;
        if (!again && h->seen.size() < 64) h->seen.push_back(key);
    }
    if (res) {
        res->vcycles = v;
        res->rel_res = r;
    }
    return st;
}

int vdi_mg_v_cycle(vdi_mg* h, const double* d_b, double* d_z) {
    if (!h || !d_b || !d_z) return VDI_ERR_INVALID_ARGUMENT;
    VDI_TRY(mg_v_cycle(h->g, h->s, d_b, d_z));
    VDI_CUDA(cudaStreamSynchronize(h->s));
    return VDI_OK;
}

int vdi_mg_residual(vdi_mg* h, const double* d_b, const double* d_z, double* d_r, double* norm) {
    if (!h || !d_b || !d_z) return VDI_ERR_INVALID_ARGUMENT;
    return mg_residual(h->g, h->s, d_b, d_z, d_r, norm);
}

int vdi_mg_apply(vdi_mg* h, const double* d_z, double* d_y) {
    if (!h || !d_z || !d_y) return VDI_ERR_INVALID_ARGUMENT;
    VDI_TRY(mg_apply(h->g, h->s, d_z, d_y));
    VDI_CUDA(cudaStreamSynchronize(h->s));
    return VDI_OK;
}

int vdi_unet_guess(vdi_unet* net, vdi_mg* h, int factor, double scale, const double* d_b, double* d_z) {
    if (!net || !h || !d_b || !d_z || (factor != 1 && factor != 2 && factor != 4 && factor != 8))
        return VDI_ERR_INVALID_ARGUMENT;
    const int kind = mg_kind(h->g);
    if (kind != VDI_MG_MAC && kind != VDI_MG_MAC_NEUMANN) {
        set_error("vdi_unet_guess: the learned guess is defined for the cell-centred MAC system");
        return VDI_ERR_INVALID_ARGUMENT;
    }
    int H, W;
    unet_dims(net, &H, &W);
    const long mn = mg_fine_size(h->g);
    cudaStream_t s = h->s;
    double* r = nullptr;
    float* io = nullptr;
    VDI_CUDA(cudaMallocAsync(&r, sizeof(double) * (mn + 1), s));
    VDI_CUDA(cudaMallocAsync(&io, sizeof(float) * 2 * size_t(H) * W, s));
    int st = mg_residual_async(h->g, s, d_b, d_z, r, r + mn);
    int m = 0, n = 0;
    if (st == VDI_OK) st = mg_dims(h->g, &m, &n);
    if (st == VDI_OK) st = unet_correct(net, s, r, r + mn, d_z, m, n, factor, scale, io, io + size_t(H) * W);
    cudaFreeAsync(io, s);
    cudaFreeAsync(r, s);
    VDI_TRY(st);
    VDI_CUDA(cudaStreamSynchronize(s));
    return VDI_OK;
}

int vdi_mg_coarse_cycle(const vdi_mg* h, int precision, int* first_level, int* ctas) {
    if (!h || !first_level || !ctas) return VDI_ERR_INVALID_ARGUMENT;
    return mg_coarse_cycle(h->g, precision, first_level, ctas);
}

int vdi_mg_tile_path(long long* persistent_launches) { return mg_tile_path(persistent_launches); }

int vdi_mg_profile(vdi_mg* h, int which, int iters, const double* d_b, double* d_z, float* ms_per_launch,
                   double* bytes_per_launch) {
    if (!h || !d_b || !d_z || !ms_per_launch || !bytes_per_launch || which < 0 || which > 6)
        return VDI_ERR_INVALID_ARGUMENT;
    return mg_profile(h->g, h->s, which, iters, d_b, d_z, ms_per_launch, bytes_per_launch);
}

int vdi_tri_solve(int n, double* d_a, double* d_b, double* d_c, double* d_d, void* stream, int* pivoted) {
    if (n < 2 || !d_a || !d_b || !d_c || !d_d) return VDI_ERR_INVALID_ARGUMENT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int* dp;
    VDI_CUDA(cudaMallocAsync(&dp, sizeof(int), s));
    VDI_TRY(launch_tri_solve(s, n, d_a, d_b, d_c, d_d, dp));
    int hp = 0;
    VDI_CUDA(cudaMemcpyAsync(&hp, dp, sizeof(int), cudaMemcpyDeviceToHost, s));
    VDI_CUDA(cudaFreeAsync(dp, s));
    VDI_CUDA(cudaStreamSynchronize(s));
    if (pivoted) *pivoted = hp > 0 ? 1 : 0;
    if (hp < 0) {
        set_error("tri_solve: zero pivot at row %d", -hp);
        return VDI_ERR_TRI_SINGULAR;
    }
    return VDI_OK;
}

}  // extern "C"

// ============================================================ autotuning
// The per-cell stencil kernels take their launch shape from the Grid, and
// each multigrid hierarchy switches from per-level tile kernels to the
// single-CTA coarse cycle below a byte threshold. Both are chosen here by
// timing the candidates with CUDA events on the simulation's own arrays; a
// process-wide cache keyed by the grid lets simulations of the same grid
// reuse a tuning.
namespace {

struct TuneKey {
    int m, n, x_sym, iv;
    bool operator<(const TuneKey& o) const {
        if (m != o.m) return m < o.m;
        if (n != o.n) return n < o.n;
        if (x_sym != o.x_sym) return x_sym < o.x_sym;
        return iv < o.iv;
    }
};

std::map<TuneKey, vdi_tune>& tune_cache() {
    static std::map<TuneKey, vdi_tune> c;
    return c;
}
std::mutex& tune_mutex() {
    static std::mutex mu;
    return mu;
}

const int BLOCK_SHAPES[][2] = {{32, 8}, {64, 4}, {128, 2}, {32, 4}, {64, 2}, {32, 16}, {64, 8}, {128, 4}, {256, 1}};
const size_t CTA_LIMITS[] = {200 * 1024, 96 * 1024, 48 * 1024, 24 * 1024, 12 * 1024, 6 * 1024};

/** Mean time of the four advection stages (idempotent as a group: each
 * repetition recomputes from u, v, p). */
int time_stencils(vdi_sim* S, double dt, float* ms) {
    cudaEvent_t e0, e1;
    VDI_CUDA(cudaEventCreate(&e0));
    VDI_CUDA(cudaEventCreate(&e1));
    auto run = [&]() -> int {
        VDI_TRY(launch_stage1(S->s, S->g, S->f, dt));
        VDI_TRY(launch_stage2(S->s, S->g, S->f));
        VDI_TRY(launch_stage34(S->s, S->g, S->f, dt));
        VDI_TRY(launch_stage5_src(S->s, S->g, S->f, S->gas, dt, S->src_mac));
        return VDI_OK;
    };
    int st = VDI_OK;
    for (int r = 0; r < 2 && st == VDI_OK; r++) st = run();
    cudaEventRecord(e0, S->s);
    for (int r = 0; r < 10 && st == VDI_OK; r++) st = run();
    cudaEventRecord(e1, S->s);
    cudaError_t e = cudaEventSynchronize(e1);
    if (st == VDI_OK && e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    VDI_TRY(st);
    VDI_CUDA(e);
    *ms /= 10;
    return VDI_OK;
}

/** Mean time of one FP64 V-cycle of system k on scratch arrays. */
int time_vcycle(vdi_sim* S, int k, const double* src, float* ms) {
    MG* g = S->mg[k];
    size_t n = size_t(mg_fine_size(g));
    double *b = nullptr, *z = nullptr;
    VDI_CUDA(cudaMalloc(&b, n * 8));
    VDI_CUDA(cudaMalloc(&z, n * 8));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st = VDI_OK;
    cudaError_t e = cudaMemcpyAsync(b, src, n * 8, cudaMemcpyDeviceToDevice, S->s);
    if (e == cudaSuccess) e = cudaMemsetAsync(z, 0, n * 8, S->s);
    for (int r = 0; r < 2 && st == VDI_OK && e == cudaSuccess; r++) st = mg_v_cycle(g, S->s, b, z);
    cudaEventRecord(e0, S->s);
    for (int r = 0; r < 8 && st == VDI_OK && e == cudaSuccess; r++) st = mg_v_cycle(g, S->s, b, z);
    cudaEventRecord(e1, S->s);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (st == VDI_OK && e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(b);
    cudaFree(z);
    VDI_TRY(st);
    VDI_CUDA(e);
    *ms /= 8;
    return VDI_OK;
}

const double* system_source(vdi_sim* S, int k) {
    return k == SOLVER_MAC ? S->src_mac : k == SOLVER_FEM ? S->src_fem : k == SOLVER_VX ? S->su : S->sv;
}

int apply_tuning(vdi_sim* S, const vdi_tune& t) {
    VDI_CUDA(cudaStreamSynchronize(S->s));
    destroy_graph(S);
    S->g.blk_x = t.blk_x;
    S->g.blk_y = t.blk_y;
    for (int k = 0; k < 4; k++)
        if (S->mg[k] && t.cta_limit[k] > 0) VDI_TRY(mg_set_cta_limit(S->mg[k], size_t(t.cta_limit[k])));
    return VDI_OK;
}

}  // namespace

int vdi_sim_autotune(vdi_sim* S, vdi_tune* out) {
    if (!S) return VDI_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(tune_mutex());
    TuneKey key{S->prm.m, S->prm.n, S->prm.x_sym, S->prm.implicit_visc};
    auto it = tune_cache().find(key);
    if (it != tune_cache().end()) {
        vdi_tune t = it->second;
        t.from_cache = 1;
        VDI_TRY(apply_tuning(S, t));
        if (out) *out = t;
        return VDI_OK;
    }
    VDI_CUDA(cudaStreamSynchronize(S->s));
    destroy_graph(S);
    // the frame timestep gives the viscous systems their hierarchy
    double dt;
    VDI_TRY(vdi_sim_timestep_select(S, S->prm.t_end / S->prm.nframes, &dt, nullptr));
    VDI_TRY(update_visc(S, dt));
    vdi_tune t{};
    float best = 1e30f;
    for (auto& b : BLOCK_SHAPES) {
        S->g.blk_x = b[0];
        S->g.blk_y = b[1];
        float ms;
        VDI_TRY(time_stencils(S, dt, &ms));
        if (ms < best * 0.98f) {
            best = ms;
            t.blk_x = b[0];
            t.blk_y = b[1];
        }
    }
    S->g.blk_x = t.blk_x;
    S->g.blk_y = t.blk_y;
    t.stencil_ms = best;
    for (int k = 0; k < 4; k++) {
        MG* g = S->mg[k];
        if (!g || mg_tiled_levels(g, VDI_MG_FP64) < 0) {
            t.tiled_levels[k] = g ? -1 : 0;
            continue;
        }
        float bk = 1e30f;
        size_t bl = mg_cta_limit(g);
        int seen = -2;
        for (size_t lim : CTA_LIMITS) {
            VDI_TRY(mg_set_cta_limit(g, lim));
            int tl = mg_tiled_levels(g, VDI_MG_FP64);
            if (tl == seen) continue;
            seen = tl;
            float ms;
            VDI_TRY(time_vcycle(S, k, system_source(S, k), &ms));
            if (ms < bk * 0.98f) {
                bk = ms;
                bl = lim;
            }
        }
        VDI_TRY(mg_set_cta_limit(g, bl));
        t.cta_limit[k] = long(bl);
        t.tiled_levels[k] = mg_tiled_levels(g, VDI_MG_FP64);
        t.vcycle_ms[k] = bk;
    }
    tune_cache()[key] = t;
    if (out) *out = t;
    return VDI_OK;
}

int vdi_sim_profile(vdi_sim* S, int which, int iters, float* ms) {
    if (!S || !ms || iters < 1 || which < 0 || which > 3) return VDI_ERR_INVALID_ARGUMENT;
    VDI_CUDA(cudaStreamSynchronize(S->s));
    double dt;
    VDI_TRY(vdi_sim_timestep_select(S, S->prm.t_end / S->prm.nframes, &dt, nullptr));
    const Grid& g = S->g;
    const int m = g.m;
    auto launch = [&]() -> int {
        switch (which) {
            case 0: return launch_advect(S->s, g, S->f, dt, S->src_mac);
            case 1:
                VDI_TRY(launch_stage1(S->s, g, S->f, dt));
                VDI_TRY(launch_stage2(S->s, g, S->f));
                VDI_TRY(launch_stage34(S->s, g, S->f, dt));
                return launch_stage5_src(S->s, g, S->f, S->gas, dt, S->src_mac);
            case 2:
                return launch_gas_update(S->s, S->gp, S->gas, S->f.u, S->f.v, m + 4, S->d_vframe, dt, S->d_time,
                                         S->gas_work, S->d_err, S->d_gstats);
            default:
                return liftoff_launch(S->s, S->gas.h, S->lcfg, S->d_lift, S->d_lhist, S->lcap, dt);
        }
    };
    if (which == 3 && S->lcfg.mode == VDI_LIFTOFF_OFF) return VDI_ERR_NOT_READY;
    VDI_TRY(launch());
    cudaEvent_t e0, e1;
    VDI_CUDA(cudaEventCreate(&e0));
    VDI_CUDA(cudaEventCreate(&e1));
    VDI_CUDA(cudaEventRecord(e0, S->s));
    int st = VDI_OK;
    for (int k = 0; k < iters && st == VDI_OK; k++) st = launch();
    VDI_CUDA(cudaEventRecord(e1, S->s));
    VDI_CUDA(cudaEventSynchronize(e1));
    float t = 0;
    VDI_CUDA(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    VDI_TRY(st);
    *ms = t / iters;
    return VDI_OK;
}

int vdi_sim_set_tuning(vdi_sim* S, const vdi_tune* t) {
    if (!S || !t || t->blk_x < 1 || t->blk_y < 1 || t->blk_x * t->blk_y > 1024) return VDI_ERR_INVALID_ARGUMENT;
    return apply_tuning(S, *t);
}

// ================================================================ batch
// Independent simulations stepped together. Each keeps its own stream and
// arrays; a timestep of the batch is one CUDA graph with one branch per
// simulation (each branch the simulation's captured step, with its own
// conditional multigrid loops), so small grids run side by side on the SMs
// and the host launches once per step.
struct vdi_batch {
    std::vector<vdi_sim*> sims;
    cudaStream_t s0 = nullptr;
    cudaEvent_t ev0 = nullptr;
    std::vector<cudaEvent_t> evd;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    std::vector<double> gdts;
};

namespace {

void batch_drop_graph(vdi_batch* B) {
    if (B->gexec) cudaGraphExecDestroy(B->gexec);
    if (B->graph) cudaGraphDestroy(B->graph);
    B->gexec = nullptr;
    B->graph = nullptr;
}

int batch_capture(vdi_batch* B, const double* dts) {
    batch_drop_graph(B);
    for (size_t k = 0; k < B->sims.size(); k++) VDI_TRY(update_visc(B->sims[k], dts[k]));
    VDI_CUDA(cudaStreamBeginCapture(B->s0, cudaStreamCaptureModeRelaxed));
    int st = VDI_OK;
    cudaError_t e = cudaEventRecord(B->ev0, B->s0);
    for (size_t k = 0; k < B->sims.size() && st == VDI_OK && e == cudaSuccess; k++) {
        vdi_sim* S = B->sims[k];
        e = cudaStreamWaitEvent(S->s, B->ev0, 0);
        if (e == cudaSuccess) st = enqueue_step(S, dts[k]);
        if (st == VDI_OK && e == cudaSuccess) e = cudaEventRecord(B->evd[k], S->s);
        if (st == VDI_OK && e == cudaSuccess) e = cudaStreamWaitEvent(B->s0, B->evd[k], 0);
    }
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(B->s0, &g);
    if (st != VDI_OK || e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (st != VDI_OK) return st;
        VDI_CUDA(e != cudaSuccess ? e : e2);
    }
    B->graph = g;
    VDI_CUDA(cudaGraphInstantiate(&B->gexec, g, 0));
    B->gdts.assign(dts, dts + B->sims.size());
    return VDI_OK;
}

}  // namespace

int vdi_batch_create(const vdi_params* prms, int count, vdi_batch** out) {
    if (!prms || count < 1 || !out) return VDI_ERR_INVALID_ARGUMENT;
    vdi_batch* B = new vdi_batch();
    auto fail = [&](int st) {
        vdi_batch_destroy(B);
        return st;
    };
    if (cudaStreamCreateWithFlags(&B->s0, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&B->ev0, cudaEventDisableTiming) != cudaSuccess)
        return fail(VDI_ERR_CUDA);
    for (int k = 0; k < count; k++) {
        vdi_sim* S = nullptr;
        int st = vdi_sim_create(prms + k, nullptr, &S);
        if (st != VDI_OK) return fail(st);
        B->sims.push_back(S);
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return fail(VDI_ERR_CUDA);
        B->evd.push_back(ev);
    }
    *out = B;
    return VDI_OK;
}

int vdi_batch_destroy(vdi_batch* B) {
    if (!B) return VDI_OK;
    if (B->s0) cudaStreamSynchronize(B->s0);
    batch_drop_graph(B);
    for (auto S : B->sims) vdi_sim_destroy(S);
    for (auto e : B->evd) cudaEventDestroy(e);
    if (B->ev0) cudaEventDestroy(B->ev0);
    if (B->s0) cudaStreamDestroy(B->s0);
    delete B;
    return VDI_OK;
}

int vdi_batch_size(const vdi_batch* B) { return B ? int(B->sims.size()) : 0; }

int vdi_batch_sim(vdi_batch* B, int k, vdi_sim** out) {
    if (!B || !out || k < 0 || k >= int(B->sims.size())) return VDI_ERR_INVALID_ARGUMENT;
    *out = B->sims[k];
    return VDI_OK;
}

int vdi_batch_init_fields(vdi_batch* B) {
    if (!B) return VDI_ERR_INVALID_ARGUMENT;
    VDI_CUDA(cudaStreamSynchronize(B->s0));
    for (auto S : B->sims) VDI_TRY(vdi_sim_init_fields(S));
    return VDI_OK;
}

int vdi_batch_autotune(vdi_batch* B, vdi_tune* out) {
    if (!B) return VDI_ERR_INVALID_ARGUMENT;
    VDI_CUDA(cudaStreamSynchronize(B->s0));
    batch_drop_graph(B);
    for (size_t k = 0; k < B->sims.size(); k++) VDI_TRY(vdi_sim_autotune(B->sims[k], out ? out + k : nullptr));
    return VDI_OK;
}

int vdi_batch_step_forward(vdi_batch* B, const double* dts, int nsteps) {
    if (!B || !dts || nsteps < 0) return VDI_ERR_INVALID_ARGUMENT;
    for (size_t k = 0; k < B->sims.size(); k++)
        if (!(dts[k] > 0)) return VDI_ERR_INVALID_ARGUMENT;
    bool same = B->gexec && std::equal(B->gdts.begin(), B->gdts.end(), dts);
    for (auto S : B->sims) destroy_graph(S);
    if (!same) VDI_TRY(batch_capture(B, dts));
    for (int q = 0; q < nsteps; q++) VDI_CUDA(cudaGraphLaunch(B->gexec, B->s0));
    VDI_CUDA(cudaStreamSynchronize(B->s0));
    for (size_t k = 0; k < B->sims.size(); k++) {
        B->sims[k]->steps += nsteps;
        int st = check_errors(B->sims[k]);
        if (st != VDI_OK) {
            std::string d = vdi_last_error();
            set_error("batch simulation %zu: %s", k, d.c_str());
            return st;
        }
    }
    return VDI_OK;
}
