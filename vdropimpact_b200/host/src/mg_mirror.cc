// The multigrid problem classes (mgs_common.cc, mgs_mac.cc, mgs_fem.cc,
// visco_impl.cc) and their solver object over the device multigrid.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>

#include <cuda_runtime.h>

#include "fluid_2d.hh"
#include "mgs_fem.hh"
#include "mgs_mac.hh"
#include "visco_impl.hh"

namespace {

double mg_rtol() {
    const char* e = getenv("VDI_MG_RTOL");
    return e ? atof(e) : 1e-10;
}

void cuda_check(cudaError_t e, const char* where) {
    if (e != cudaSuccess) {
        char msg[512];
        snprintf(msg, sizeof(msg), "%s: %s", where, cudaGetErrorString(e));
        fatal_error(msg, 1);
    }
}

}  // namespace

// ------------------------------------------------------------ mgs_common
mgs_common::mgs_common(int m_, int n_)
    : m(m_), n(n_), mn(m_ * n_), scount(0), t_prev(0), t0(0), z_prev(new double[mn]()), z(new double[mn]()),
      wc_time(0.), tp() {}

mgs_common::~mgs_common() {
    delete[] z;
    delete[] z_prev;
}

void mgs_common::initial_guess(double t) {
    // mgs_common.cc:17-50: store the first two solutions, then extrapolate
    // linearly in time from the last two
    if (scount < 2) {
        if (scount == 1) {
            memcpy(z_prev, z, mn * sizeof(double));
            t0 = t;
        } else t_prev = t;
        scount++;
    } else {
        if (fabs(t0 - t_prev) < std::numeric_limits<double>::epsilon() * 10) {
            fputs("Multigrid routine called for duplicate times\n", stderr);
            return;
        }
        double a = 1. / (t0 - t_prev), b = (t - t_prev) * a, c = (t - t0) * a;
        for (int ij = 0; ij < mn; ij++) {
            double zz = z[ij];
            z[ij] = b * zz - c * z_prev[ij];
            z_prev[ij] = zz;
        }
        t_prev = t0;
        t0 = t;
    }
}

// ------------------------------------------------------------ solver object
vdi_tgmg_core::vdi_tgmg_core(int kind_, int m_, int n_, double* b_, double* z_)
    : kind(kind_), m(m_), n(n_), mn(m_ * n_), b(b_), z(z_), h(NULL), d_b(NULL), d_z(NULL) {
    cuda_check(cudaMalloc(&d_b, mn * sizeof(double)), "cudaMalloc");
    cuda_check(cudaMalloc(&d_z, mn * sizeof(double)), "cudaMalloc");
}

vdi_tgmg_core::~vdi_tgmg_core() {
    if (h) vdi_mg_destroy(h);
    cudaFree(d_b);
    cudaFree(d_z);
}

void vdi_tgmg_core::setup(double c1, double c2, int x_sym) {
    if (h) vdi_mg_destroy(h);
    h = NULL;
    vdi_check(vdi_mg_create(kind, m, n, c1, c2, x_sym, NULL, &h), "vdi_mg_create");
}

void vdi_tgmg_core::clear_z() { memset(z, 0, mn * sizeof(double)); }

void vdi_tgmg_core::push() {
    if (!h) fatal_error("multigrid used before setup()", 1);
    cuda_check(cudaMemcpy(d_b, b, mn * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    cuda_check(cudaMemcpy(d_z, z, mn * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
}

void vdi_tgmg_core::pull() {
    cuda_check(cudaMemcpy(z, d_z, mn * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
}

bool vdi_tgmg_core::solve_v_cycle(tgmg_predict& tp) {
    push();
    vdi_mg_result r;
    int st = vdi_mg_solve(h, d_b, d_z, mg_rtol(), 200, VDI_MG_FP64, &r);
    pull();
    if (st == VDI_ERR_MG_NOT_CONVERGED) return false;
    vdi_check(st, "vdi_mg_solve");
    tp.record(r.vcycles);
    return true;
}

void vdi_tgmg_core::v_cycle() {
    push();
    vdi_check(vdi_mg_v_cycle(h, d_b, d_z), "vdi_mg_v_cycle");
    pull();
}

void vdi_tgmg_core::residual(double* r) {
    push();
    double* d_r;
    double nrm;
    cuda_check(cudaMalloc(&d_r, mn * sizeof(double)), "cudaMalloc");
    vdi_check(vdi_mg_residual(h, d_b, d_z, d_r, &nrm), "vdi_mg_residual");
    cuda_check(cudaMemcpy(r, d_r, mn * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    cudaFree(d_r);
}

void vdi_tgmg_core::output(const char* filename, double* data, double ax, double dx, double ay, double dy) {
    FILE* f = safe_fopen(filename, "wb");
    std::vector<float> row(m + 1);
    row[0] = float(m);
    for (int i = 0; i < m; i++) row[i + 1] = float(ax + i * dx);
    fwrite(row.data(), sizeof(float), m + 1, f);
    for (int j = 0; j < n; j++) {
        row[0] = float(ay + j * dy);
        for (int i = 0; i < m; i++) row[i + 1] = float(data[i + m * j]);
        fwrite(row.data(), sizeof(float), m + 1, f);
    }
    fclose(f);
}

void vdi_tgmg_core::output_res(const char* filename, double ax, double dx, double ay, double dy) {
    std::vector<double> r(mn);
    residual(r.data());
    output(filename, r.data(), ax, dx, ay, dy);
}

// ------------------------------------------------------------ problem classes
// The diagonal reciprocals of the MAC stencil: interior columns with the
// bottom, middle and top rows, then the side columns with the same rows.
#define VDI_MAC_RECIPROCALS                                                                  \
    cc0(-1. / (2 * xxsp + 3 * yysp)), cc1(-1. / (2 * xxsp + 2 * yysp)), cc2(-1. / (2 * xxsp + yysp)), \
    cc3(-1. / (xxsp + 3 * yysp)), cc4(-1. / (xxsp + 2 * yysp)), cc5(-1. / (xxsp + yysp))

mgs_mac::mgs_mac(fluid_2d& f)
    : mgs_common(f.m, f.n), xxsp(f.xxsp), yysp(f.yysp), VDI_MAC_RECIPROCALS,
      acc(tgmg_accuracy(2 * (xxsp + yysp) * f.dt_reg, 1e6)), mg(*this, f.src, z), dx_(f.dx), dy_(f.dy) {
    mg.setup();
    mg.clear_z();
}

mgs_mac::mgs_mac(int m_, int n_, double dx, double dy, double* b)
    : mgs_common(m_, n_), xxsp(1. / (dx * dx)), yysp(1. / (dy * dy)), VDI_MAC_RECIPROCALS,
      acc(tgmg_accuracy(2 * (xxsp + yysp), 1e6)), mg(*this, b, z), dx_(dx), dy_(dy) {}

#undef VDI_MAC_RECIPROCALS

void mgs_mac::solve_v_cycle() {
    double t0 = wtime();
    if (!mg.solve_v_cycle(tp)) failure();
    wc_time += wtime() - t0;
}

// The bilinear element's stencil terms from the spacing ratios.
#define VDI_FEM_TERMS                                                                              \
    dydx(dy / dx), dxdy(dx / dy), fm(4. / 3. * (dxdy + dydx)), fm_inv(1.0 / fm),                    \
    fey(1. / 3. * (-2 * dxdy + dydx)), hey(0.5 * fey), fex(1. / 3. * (-2 * dydx + dxdy)), hex(0.5 * fex), \
    fc(-1. / 6. * (dxdy + dydx))

mgs_fem::mgs_fem(fluid_2d& f)
    : mgs_common(f.me, f.ne), dydx(f.dy / f.dx), dxdy(f.dx / f.dy), fm(4. / 3. * (dxdy + dydx)), fm_inv(1.0 / fm),
      fey(1. / 3. * (-2 * dxdy + dydx)), hey(0.5 * fey), fex(1. / 3. * (-2 * dydx + dxdy)), hex(0.5 * fex),
      fc(-1. / 6. * (dxdy + dydx)), acc(tgmg_accuracy(fm, 1e8)), mg(*this, f.src, z), dx_(f.dx), dy_(f.dy) {
    mg.setup();
    mg.clear_z();
}

mgs_fem::mgs_fem(int m_, int n_, double dx, double dy, double* b)
    : mgs_common(m_, n_), VDI_FEM_TERMS, acc(tgmg_accuracy(fm, 1e8)), mg(*this, b, z), dx_(dx), dy_(dy) {}

#undef VDI_FEM_TERMS

double mgs_fem::mul_a(int i, int ij) {
    if (ij < m) return 0;   // the Dirichlet bottom row
    const double* w = z + ij;
    const double* wd = w - m;
    const bool top = ij >= mn - m;
    // the row below always couples; the row above only off the top edge,
    // where the side couplings take the full weight fex instead of hex
    if (i == 0) {
        return top ? fc * wd[1] + hey * (*wd) + hex * w[1]
                   : fc * (wd[1] + w[m + 1]) + hey * (*wd + w[m]) + fex * w[1];
    }
    if (i == m - 1) {
        return top ? fc * wd[-1] + hey * (*wd) + hex * w[-1]
                   : fc * (wd[-1] + w[m - 1]) + hey * (*wd + w[m]) + fex * w[-1];
    }
    return top ? fc * (wd[-1] + wd[1]) + fey * (*wd) + hex * (w[-1] + w[1])
               : fc * (wd[-1] + wd[1] + w[m - 1] + w[m + 1]) + fey * (*wd + w[m]) + fex * (w[-1] + w[1]);
}

void mgs_fem::solve_v_cycle() {
    double t0 = wtime();
    if (!mg.solve_v_cycle(tp)) failure();
    wc_time += wtime() - t0;
}

visco_impl::visco_impl(fluid_2d& f, bool horizontal_vel_)
    : mgs_common(f.m, f.n), x_sym(f.x_sym), horizontal_vel(horizontal_vel_), acc(tgmg_accuracy(1., 1e3)), vfx(0.),
      vfy(0.), mg(*this, f.src, z) {}

void visco_impl::setup_and_solve(double vfx_, double vfy_, double t) {
    double t0 = wtime();
    if (fabs(vfx_ - vfx) > 1e2 * std::numeric_limits<double>::epsilon() * vfx || vfx == 0) {
        vfx = vfx_;
        vfy = vfy_;
        mg.setup();
    }
    initial_guess(t);
    if (!mg.solve_v_cycle(tp)) {
        fputs("Multigrid routine for implicit viscosity failed\n", stderr);
        exit(1);
    }
    wc_time += wtime() - t0;
}
