// Stencil kernels of one timestep of fluid_2d::step_forward
// (fluid_2d.cc:93-405) and the boundary conditions of fluid_2d_sio.cc.
//
// Every field lives in its own FP64 array over the ghosted grid: (n+4) rows
// of pitch P = m+4, cell (i,j) at (j+2)*P + i+2, i in [-2,m+1], j in [-2,n+1].
// Expressions keep the reference's evaluation order; this file is compiled
// with -fmad=false so that, given the same inputs, the results equal the
// reference's double-precision results bit for bit.
#include "step_kernels.hh"

#include <algorithm>

#include <cmath>

namespace vdi {

__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }

// fluid_2d.cc:445-449
__device__ __forceinline__ double delta_lim(double f0, double f1, double f2) {
    double drm = f1 - f0, drp = f2 - f1;
    return drm > 0 ? (drp > 0 ? 2 * dmin(drm, drp) : 0) : (drp > 0 ? 0 : -2 * dmax(drm, drp));
}
// fluid_2d.cc:434-437
__device__ __forceinline__ double delta_f(double f0, double f1, double f2) {
    double drc = 0.5 * (f2 - f0);
    return drc > 0 ? dmin(drc, delta_lim(f0, f1, f2)) : dmax(drc, -delta_lim(f0, f1, f2));
}
// fluid_2d.cc:422-426
__device__ __forceinline__ double mono_diff(double f0, double f1, double f2, double f3, double f4) {
    double tdrc = f3 - f1, s = (1 / 6.) * (4 * tdrc - delta_f(f0, f1, f2) - delta_f(f2, f3, f4)),
           t = delta_lim(f1, f2, f3);
    return tdrc > 0 ? dmin(s, t) : dmax(s, -t);
}
// fluid_2d.cc:455-461
__device__ __forceinline__ void godunov_set(double u0, double& u1, double v0, double& v1) {
    if (u0 > -u1) {
        if (u0 > 0) {
            u1 = u0;
            v1 = v0;
            return;
        }
    } else if (u1 < 0)
        return;
    u1 = 0;
    v1 = 0.5 * (v0 + v1);
}
// fluid_2d.cc:469-476
__device__ __forceinline__ void godunov_set_tang(double& u0, double& u1, double v0, double& v1) {
    if (u0 > -u1) {
        if (u0 > 0) {
            u1 = u0;
            v1 = v0;
            return;
        }
    } else if (u1 < 0) {
        u0 = u1;
        return;
    }
    v1 = 0.5 * (v0 + v1);
    u0 = 0.5 * (u0 + u1);
    u1 = 0;
}

#define CELL_LOOP                                                    \
    int i = blockIdx.x * blockDim.x + threadIdx.x;                   \
    int j = blockIdx.y * blockDim.y + threadIdx.y;                   \
    if (i >= g.m || j >= g.n) return;                                \
    const int P = g.m + 4;                                           \
    const int c = (j + 2) * P + i + 2;

// -------------------------------------------------------------- stage 1
// fluid_2d.cc:105-132, then zero_edge_velocities (fluid_2d.cc:480-482)
__global__ void k_stage1(Grid g, Fields f, double dt) {
    CELL_LOOP
    const double* u = f.u;
    const double* v = f.v;
    double uc = u[c], vc = v[c];
    double uy = g.ysp * mono_diff(u[c - 2 * P], u[c - P], uc, u[c + P], u[c + 2 * P]);
    double vy = g.ysp * mono_diff(v[c - 2 * P], v[c - P], vc, v[c + P], v[c + 2 * P]);
    double ux = g.xsp * mono_diff(u[c - 2], u[c - 1], uc, u[c + 1], u[c + 2]);
    double vx = g.xsp * mono_diff(v[c - 2], v[c - 1], vc, v[c + 1], v[c + 2]);
    f.uy[c] = uy; f.vy[c] = vy; f.ux[c] = ux; f.vx[c] = vx;
    f.ud[c] = uc - 0.5 * (g.dy + dt * vc) * uy;
    f.vd[c] = vc - 0.5 * (g.dy + dt * vc) * vy;
    f.ul[c] = (g.x_sym && i == 0) ? 0. : uc - 0.5 * (g.dx + dt * uc) * ux;
    f.vl[c] = vc - 0.5 * (g.dx + dt * uc) * vx;
    f.ur[c] = uc + 0.5 * (g.dx - dt * uc) * ux;
    f.vr[c] = vc + 0.5 * (g.dx - dt * uc) * vx;
    f.uu[c] = uc + 0.5 * (g.dy - dt * vc) * uy;
    f.vu[c] = vc + 0.5 * (g.dy - dt * vc) * vy;
}

// -------------------------------------------------------------- stage 2
// fluid_2d.cc:137-150. Each edge value is written by exactly one thread.
__global__ void k_stage2(Grid g, Fields f) {
    CELL_LOOP
    if (i < g.m - 1) {
        double u0 = f.ur[c], u1 = f.ul[c + 1], v1 = f.vl[c + 1];
        godunov_set_tang(u0, u1, f.vr[c], v1);
        f.ur[c] = u0; f.ul[c + 1] = u1; f.vl[c + 1] = v1;
        if (i == 0) f.ur[c - 1] = f.ul[c];
    } else {
        f.ul[c + 1] = f.ur[c];
        f.vl[c + 1] = f.vr[c];
    }
    if (j < g.n - 1) {
        double u0 = f.vu[c], u1 = f.vd[c + P], v1 = f.ud[c + P];
        godunov_set_tang(u0, u1, f.uu[c], v1);
        f.vu[c] = u0; f.vd[c + P] = u1; f.ud[c + P] = v1;
        if (j == 0) f.vu[c - P] = f.vd[c];
    } else {
        f.vd[c + P] = f.vu[c];
        f.ud[c + P] = f.uu[c];
    }
}

// ---------------------------------------------------------- stages 3-4
// fluid_2d.cc:153-201: transverse terms, then half-step edge velocities and
// the viscous force (written to the second edge set and fc0/fc1).
__global__ void k_stage34(Grid g, Fields f, double dt) {
    CELL_LOOP
    double c0 = 0.5 * g.xsp * (f.ul[c + 1] + f.ul[c]) * (f.ur[c] - f.ur[c - 1]);
    double c1 = 0.5 * g.xsp * (f.ul[c + 1] + f.ul[c]) * (f.vl[c + 1] - f.vl[c]);
    double c2 = 0.5 * g.ysp * (f.vd[c + P] + f.vd[c]) * (f.ud[c + P] - f.ud[c]);
    double c3 = 0.5 * g.ysp * (f.vd[c + P] + f.vd[c]) * (f.vu[c] - f.vu[c - P]);
    const double* u = f.u;
    const double* v = f.v;
    const double* p = f.p;
    double uc = u[c], vc = v[c];
    double px = 0.5 * g.xsp * (p[c + P + 1] + p[c + 1] - p[c + P] - p[c]);
    double py = 0.5 * g.ysp * (p[c + P + 1] - p[c + 1] + p[c + P] - p[c]);
    // centered_diff, fluid_2d.cc:412-417
    double uyy = g.yysp * (u[c - P] - 2 * uc + u[c + P]);
    double vyy = g.yysp * (v[c - P] - 2 * vc + v[c + P]);
    double uxx = g.xxsp * (u[c - 1] - 2 * uc + u[c + 1]);
    double vxx = g.xxsp * (v[c - 1] - 2 * vc + v[c + 1]);
    double f_x = -px * g.rhoinv + g.viscfac * (uxx + uyy);
    double f_y = -py * g.rhoinv + g.viscfac * (vxx + vyy);
    double ux = f.ux[c], uy = f.uy[c], vx = f.vx[c], vy = f.vy[c];
    f.ud2[c] = uc + 0.5 * (-g.dy * uy + dt * (-c0 - vc * uy + f_x));
    f.vd2[c] = vc + 0.5 * (-g.dy * vy + dt * (-c1 - vc * vy + f_y));
    f.ul2[c] = uc + 0.5 * (-g.dx * ux + dt * (-uc * ux - c2 + f_x));
    f.vl2[c] = vc + 0.5 * (-g.dx * vx + dt * (-uc * vx - c3 + f_y));
    f.ur2[c] = uc + 0.5 * (g.dx * ux + dt * (-uc * ux - c2 + f_x));
    f.vr2[c] = vc + 0.5 * (g.dx * vx + dt * (-uc * vx - c3 + f_y));
    f.uu2[c] = uc + 0.5 * (g.dy * uy + dt * (-c0 - vc * uy + f_x));
    f.vu2[c] = vc + 0.5 * (g.dy * vy + dt * (-c1 - vc * vy + f_y));
    f.fc0[c] = g.viscfac * (uxx + uyy);
    f.fc1[c] = g.viscfac * (vxx + vyy);
}

// ---------------------------------------------------------- stage 5 + 6
// fluid_2d.cc:205-232: zero_edge_velocities, normal upwinding, and the MAC
// source with the bottom Dirichlet term. Every thread recomputes the
// upwinded values of its own four edges from the stage-4 set, writes the
// left and bottom ones (and the ghost ones at the right and top), and forms
// the divergence.
__global__ void k_stage5_src(Grid g, Fields f, Gas gs, double dt, double* __restrict__ src) {
    CELL_LOOP
    // left edge of (i,j)
    double ulL, vlL;
    if (i == 0) {
        ulL = g.x_sym ? 0. : f.ul2[c];
        vlL = f.vl2[c];
    } else {
        ulL = f.ul2[c];
        vlL = f.vl2[c];
        godunov_set(f.ur2[c - 1], ulL, f.vr2[c - 1], vlL);
    }
    // right edge
    double ulR, vlR;
    if (i < g.m - 1) {
        ulR = f.ul2[c + 1];
        vlR = f.vl2[c + 1];
        godunov_set(f.ur2[c], ulR, f.vr2[c], vlR);
    } else {
        ulR = f.ur2[c];
        vlR = f.vr2[c];
        f.ul[c + 1] = ulR;
        f.vl[c + 1] = vlR;
    }
    // bottom edge
    double vdB, udB;
    if (j == 0) {
        vdB = f.vd2[c];
        udB = f.ud2[c];
    } else {
        vdB = f.vd2[c];
        udB = f.ud2[c];
        godunov_set(f.vu2[c - P], vdB, f.uu2[c - P], udB);
    }
    // top edge
    double vdT, udT;
    if (j < g.n - 1) {
        vdT = f.vd2[c + P];
        udT = f.ud2[c + P];
        godunov_set(f.vu2[c], vdT, f.uu2[c], udT);
    } else {
        vdT = f.vu2[c];
        udT = f.uu2[c];
        f.vd[c + P] = vdT;
        f.ud[c + P] = udT;
    }
    f.ul[c] = ulL; f.vl[c] = vlL; f.vd[c] = vdB; f.ud[c] = udB;
    double s = g.xsp * (ulR - ulL) + g.ysp * (vdT - vdB);
    if (j == 0) {
        const double macfac = 0.125 * g.rhoinv * dt;
        double sbc = macfac * (gs.gp_old[i] + gs.gp_old[i + 1] + gs.gp[i] + gs.gp[i + 1]);
        s -= 2 * g.yysp * sbc;
    }
    src[i + g.m * j] = s;
}

// ------------------------------------------------ fused stages 1 to 5
// k_stage1, k_stage2, k_stage34 and k_stage5_src (fluid_2d.cc:105-232) as
// one kernel: a CTA loads u, v and p around a TX x TY tile once and carries
// the stages through shared memory, each stage on a region one cell smaller
// than the previous one's (stage 1 on the tile grown by two cells left and
// below and three right and above, stage 2 by two/two, stages 3-4 by one).
// It writes only what the rest of the step reads: the final edge velocities
// ul, vl, vd, ud (with the ghost edges at the right and top), the viscous
// force fc0, fc1 and the MAC source. Stage 1 parks each cell's four limited
// slopes in the stage-4 arrays, which stage 4 reads before it overwrites them.
// The source's bottom-row gas-pressure
// term depends on the gas layer, which runs concurrently, so
// k_mac_src_bottom adds it after the two streams join. Every value is
// computed by the same expressions as in the four kernels, so the results
// are bit-identical.
namespace {
constexpr int ADV_TX = 32, ADV_TY = 16;
constexpr int ADV_W = ADV_TX + 4, ADV_H = ADV_TY + 4, ADV_N = ADV_W * ADV_H;   // edge windows
// threads of a CTA: at least one per edge-window cell, so each stage is one
// pass (23 warps; stage 5 uses the first TX x TY of them)
constexpr int ADV_NT = (ADV_N + 31) / 32 * 32;
static_assert(ADV_NT >= ADV_TX * ADV_TY, "stage 5 takes one tile cell per thread");
constexpr int ADV_UW = ADV_TX + 8, ADV_UH = ADV_TY + 8;                        // u, v window
constexpr int ADV_PW = ADV_TX + 3, ADV_PH = ADV_TY + 3;                        // pressure nodes
constexpr size_t ADV_SMEM = (size_t(16) * ADV_N + 2 * ADV_UW * ADV_UH + ADV_PW * ADV_PH) * sizeof(double);
}  // namespace

__global__ void __launch_bounds__(ADV_NT) k_advect(Grid g, Fields f, double dt, double* __restrict__ src) {
    extern __shared__ __align__(16) double asm_[];
    double* E = asm_;                                  // 8 edge sets of stages 1-2: ud vd ul vl ur vr uu vu
    double* E2 = E + 8 * ADV_N;                        // 8 edge sets of stage 4
    double* U = E2 + 8 * ADV_N;
    double* Vv = U + ADV_UW * ADV_UH;
    double* Pn = Vv + ADV_UW * ADV_UH;
    double *sud = E, *svd = E + ADV_N, *sul = E + 2 * ADV_N, *svl = E + 3 * ADV_N, *sur = E + 4 * ADV_N,
           *svr = E + 5 * ADV_N, *suu = E + 6 * ADV_N, *svu = E + 7 * ADV_N;
    double *sud2 = E2, *svd2 = E2 + ADV_N, *sul2 = E2 + 2 * ADV_N, *svl2 = E2 + 3 * ADV_N, *sur2 = E2 + 4 * ADV_N,
           *svr2 = E2 + 5 * ADV_N, *suu2 = E2 + 6 * ADV_N, *svu2 = E2 + 7 * ADV_N;
    const int m = g.m, n = g.n, P = m + 4;
    const int x0 = blockIdx.x * ADV_TX, y0 = blockIdx.y * ADV_TY;
    const int ox = x0 - 2, oy = y0 - 2;                // window cell (0,0)
    const int tid = threadIdx.x;
    // u, v over cells [x0-4, x0+TX+3] x [y0-4, y0+TY+3], inside the ghost layers
    for (int t = tid; t < ADV_UW * ADV_UH; t += ADV_NT) {
        const int i = x0 - 4 + t % ADV_UW, j = y0 - 4 + t / ADV_UW;
        const bool in = i >= -2 && i <= m + 1 && j >= -2 && j <= n + 1;
        const int c = (j + 2) * P + i + 2;
        U[t] = in ? f.u[c] : 0.;
        Vv[t] = in ? f.v[c] : 0.;
    }
    for (int t = tid; t < ADV_PW * ADV_PH; t += ADV_NT) {
        const int i = x0 - 1 + t % ADV_PW, j = y0 - 1 + t / ADV_PW;
        const bool in = i >= -2 && i <= m + 1 && j >= -2 && j <= n + 1;
        Pn[t] = in ? f.p[(j + 2) * P + i + 2] : 0.;
    }
    __syncthreads();
    auto uat = [&](int i, int j) { return U[(j - y0 + 4) * ADV_UW + (i - x0 + 4)]; };
    auto vat = [&](int i, int j) { return Vv[(j - y0 + 4) * ADV_UW + (i - x0 + 4)]; };
    auto pat = [&](int i, int j) { return Pn[(j - y0 + 1) * ADV_PW + (i - x0 + 1)]; };
    // ---- stage 1 (k_stage1) on window cells [0, W) x [0, H)
    for (int t = tid; t < ADV_N; t += ADV_NT) {
        const int a = t % ADV_W, b = t / ADV_W, i = ox + a, j = oy + b;
        if (i < 0 || i >= m || j < 0 || j >= n) continue;
        double uc = uat(i, j), vc = vat(i, j);
        double uy = g.ysp * mono_diff(uat(i, j - 2), uat(i, j - 1), uc, uat(i, j + 1), uat(i, j + 2));
        double vy = g.ysp * mono_diff(vat(i, j - 2), vat(i, j - 1), vc, vat(i, j + 1), vat(i, j + 2));
        double ux = g.xsp * mono_diff(uat(i - 2, j), uat(i - 1, j), uc, uat(i + 1, j), uat(i + 2, j));
        double vx = g.xsp * mono_diff(vat(i - 2, j), vat(i - 1, j), vc, vat(i + 1, j), vat(i + 2, j));
        // the slopes wait for stage 4 in its own arrays, free until then
        sul2[t] = ux; sud2[t] = uy; svl2[t] = vx; svd2[t] = vy;
        sud[t] = uc - 0.5 * (g.dy + dt * vc) * uy;
        svd[t] = vc - 0.5 * (g.dy + dt * vc) * vy;
        sul[t] = (g.x_sym && i == 0) ? 0. : uc - 0.5 * (g.dx + dt * uc) * ux;
        svl[t] = vc - 0.5 * (g.dx + dt * uc) * vx;
        sur[t] = uc + 0.5 * (g.dx - dt * uc) * ux;
        svr[t] = vc + 0.5 * (g.dx - dt * uc) * vx;
        suu[t] = uc + 0.5 * (g.dy - dt * vc) * uy;
        svu[t] = vc + 0.5 * (g.dy - dt * vc) * vy;
    }
    __syncthreads();
    // ---- stage 2 (k_stage2) on window cells [0, W-1) x [0, H-1)
    for (int t = tid; t < ADV_N; t += ADV_NT) {
        const int a = t % ADV_W, b = t / ADV_W, i = ox + a, j = oy + b;
        if (a >= ADV_W - 1 || b >= ADV_H - 1 || i < 0 || i >= m || j < 0 || j >= n) continue;
        if (i < m - 1) {
            double u0 = sur[t], u1 = sul[t + 1], v1 = svl[t + 1];
            godunov_set_tang(u0, u1, svr[t], v1);
            sur[t] = u0; sul[t + 1] = u1; svl[t + 1] = v1;
            if (i == 0) sur[t - 1] = sul[t];
        } else {
            sul[t + 1] = sur[t];
            svl[t + 1] = svr[t];
        }
        if (j < n - 1) {
            double u0 = svu[t], u1 = svd[t + ADV_W], v1 = sud[t + ADV_W];
            godunov_set_tang(u0, u1, suu[t], v1);
            svu[t] = u0; svd[t + ADV_W] = u1; sud[t + ADV_W] = v1;
            if (j == 0) svu[t - ADV_W] = svd[t];
        } else {
            svd[t + ADV_W] = svu[t];
            sud[t + ADV_W] = suu[t];
        }
    }
    __syncthreads();
    // ---- stages 3-4 (k_stage34) on window cells [1, W-1) x [1, H-1)
    for (int t = tid; t < ADV_N; t += ADV_NT) {
        const int a = t % ADV_W, b = t / ADV_W, i = ox + a, j = oy + b;
        if (a < 1 || a >= ADV_W - 1 || b < 1 || b >= ADV_H - 1 || i < 0 || i >= m || j < 0 || j >= n) continue;
        double c0 = 0.5 * g.xsp * (sul[t + 1] + sul[t]) * (sur[t] - sur[t - 1]);
        double c1 = 0.5 * g.xsp * (sul[t + 1] + sul[t]) * (svl[t + 1] - svl[t]);
        double c2 = 0.5 * g.ysp * (svd[t + ADV_W] + svd[t]) * (sud[t + ADV_W] - sud[t]);
        double c3 = 0.5 * g.ysp * (svd[t + ADV_W] + svd[t]) * (svu[t] - svu[t - ADV_W]);
        double uc = uat(i, j), vc = vat(i, j);
        double px = 0.5 * g.xsp * (pat(i + 1, j + 1) + pat(i + 1, j) - pat(i, j + 1) - pat(i, j));
        double py = 0.5 * g.ysp * (pat(i + 1, j + 1) - pat(i + 1, j) + pat(i, j + 1) - pat(i, j));
        double uyy = g.yysp * (uat(i, j - 1) - 2 * uc + uat(i, j + 1));
        double vyy = g.yysp * (vat(i, j - 1) - 2 * vc + vat(i, j + 1));
        double uxx = g.xxsp * (uat(i - 1, j) - 2 * uc + uat(i + 1, j));
        double vxx = g.xxsp * (vat(i - 1, j) - 2 * vc + vat(i + 1, j));
        double f_x = -px * g.rhoinv + g.viscfac * (uxx + uyy);
        double f_y = -py * g.rhoinv + g.viscfac * (vxx + vyy);
        // this cell's slopes from stage 1, read before its stage-4 values
        // overwrite them
        double ux = sul2[t], uy = sud2[t], vx = svl2[t], vy = svd2[t];
        sud2[t] = uc + 0.5 * (-g.dy * uy + dt * (-c0 - vc * uy + f_x));
        svd2[t] = vc + 0.5 * (-g.dy * vy + dt * (-c1 - vc * vy + f_y));
        sul2[t] = uc + 0.5 * (-g.dx * ux + dt * (-uc * ux - c2 + f_x));
        svl2[t] = vc + 0.5 * (-g.dx * vx + dt * (-uc * vx - c3 + f_y));
        sur2[t] = uc + 0.5 * (g.dx * ux + dt * (-uc * ux - c2 + f_x));
        svr2[t] = vc + 0.5 * (g.dx * vx + dt * (-uc * vx - c3 + f_y));
        suu2[t] = uc + 0.5 * (g.dy * uy + dt * (-c0 - vc * uy + f_x));
        svu2[t] = vc + 0.5 * (g.dy * vy + dt * (-c1 - vc * vy + f_y));
        if (a >= 2 && a < ADV_TX + 2 && b >= 2 && b < ADV_TY + 2) {
            const int c = (j + 2) * P + i + 2;
            f.fc0[c] = g.viscfac * (uxx + uyy);
            f.fc1[c] = g.viscfac * (vxx + vyy);
        }
    }
    __syncthreads();
    // ---- stage 5 (k_stage5_src without the bottom gas term) on the tile
    {
        if (tid >= ADV_TX * ADV_TY) return;
        const int a = 2 + tid % ADV_TX, b = 2 + tid / ADV_TX, i = ox + a, j = oy + b;
        if (i >= m || j >= n) return;
        const int t = b * ADV_W + a;
        const int c = (j + 2) * P + i + 2;
        double ulL, vlL;
        if (i == 0) {
            ulL = g.x_sym ? 0. : sul2[t];
            vlL = svl2[t];
        } else {
            ulL = sul2[t];
            vlL = svl2[t];
            godunov_set(sur2[t - 1], ulL, svr2[t - 1], vlL);
        }
        double ulR, vlR;
        if (i < m - 1) {
            ulR = sul2[t + 1];
            vlR = svl2[t + 1];
            godunov_set(sur2[t], ulR, svr2[t], vlR);
        } else {
            ulR = sur2[t];
            vlR = svr2[t];
            f.ul[c + 1] = ulR;
            f.vl[c + 1] = vlR;
        }
        double vdB, udB;
        if (j == 0) {
            vdB = svd2[t];
            udB = sud2[t];
        } else {
            vdB = svd2[t];
            udB = sud2[t];
            godunov_set(svu2[t - ADV_W], vdB, suu2[t - ADV_W], udB);
        }
        double vdT, udT;
        if (j < n - 1) {
            vdT = svd2[t + ADV_W];
            udT = sud2[t + ADV_W];
            godunov_set(svu2[t], vdT, suu2[t], udT);
        } else {
            vdT = svu2[t];
            udT = suu2[t];
            f.vd[c + P] = vdT;
            f.ud[c + P] = udT;
        }
        f.ul[c] = ulL; f.vl[c] = vlL; f.vd[c] = vdB; f.ud[c] = udB;
        src[i + g.m * j] = g.xsp * (ulR - ulL) + g.ysp * (vdT - vdB);
    }
}

/** The bottom-row term of the MAC source (fluid_2d.cc:228-232), added once
 * the gas layer has updated gp. */
__global__ void k_mac_src_bottom(Grid g, Gas gs, double dt, double* __restrict__ src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.m) return;
    const double macfac = 0.125 * g.rhoinv * dt;
    double sbc = macfac * (gs.gp_old[i] + gs.gp_old[i + 1] + gs.gp[i] + gs.gp[i + 1]);
    double s = src[i];
    s -= 2 * g.yysp * sbc;
    src[i] = s;
}

// ------------------------------------------- MAC correction + advection
// fluid_2d.cc:236-261, with the corrected edge velocities formed on the fly.
// Also advances the simulation time by dt/2 (fluid_2d.cc:251).
__global__ void k_mac_advect(Grid g, Fields f, Gas gs, const double* __restrict__ q, double dt, double* d_time) {
    CELL_LOOP
    const int m = g.m;
    const int ij = i + m * j;
    double ulL = f.ul[c];
    if (i >= 1) ulL -= (q[ij] - q[ij - 1]) * g.xsp;
    double ulR = f.ul[c + 1];
    if (i + 1 <= m - 1) ulR -= (q[ij + 1] - q[ij]) * g.xsp;
    double vdB = f.vd[c];
    if (j >= 1) {
        vdB -= (q[ij] - q[ij - m]) * g.ysp;
    } else {
        const double macfac = 0.125 * g.rhoinv * dt;
        double sbc = macfac * (gs.gp_old[i] + gs.gp_old[i + 1] + gs.gp[i] + gs.gp[i + 1]);
        vdB -= 2 * g.ysp * (q[ij] - sbc);
    }
    double vdT = f.vd[c + P];
    if (j + 1 <= g.n - 1) vdT -= (q[ij + m] - q[ij]) * g.ysp;
    double uc = f.u[c], vc = f.v[c];
    f.fc0[c] = uc + dt * (-0.5 * (g.xsp * (ulR + ulL) * (ulR - ulL) + g.ysp * (vdT + vdB) * (f.ud[c + P] - f.ud[c])) +
                          f.fc0[c]);
    f.fc1[c] = vc + dt * (-0.5 * (g.xsp * (ulR + ulL) * (f.vl[c + 1] - f.vl[c]) + g.ysp * (vdT + vdB) * (vdT - vdB)) +
                          f.fc1[c]);
    if (i == 0 && j == 0) *d_time += 0.5 * dt;
}

// -------------------------------------------------- inviscid boundaries
// fluid_2d_sio.cc:256-290 and 366-405: far-field ghost velocities stepped
// with a composite Simpson integral of the base pressure. One warp per ghost
// point; lanes split the quadrature nodes and reduce with shuffles.
__global__ void k_inviscid_bc(Grid g, Fields f, Gas gs, double dt) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    const int m = g.m, n = g.n, ml = m + 4, P = m + 4, me = m + 1;
    int total = 2 * n + 2 * ml;
    if (warp >= total) return;
    double x, y;
    int idx;     // ghosted array index of the ghost cell
    int right_row = -1;
    if (warp < 2 * n) {
        int j = warp >> 1, outer = warp & 1;
        x = g.bx + g.dx * (outer ? 1.5 : 0.5);
        y = g.ay + (j + 0.5) * g.dy;
        idx = (j + 2) * P + m + 2 + outer;
        right_row = j;
    } else {
        int k = warp - 2 * n;
        int col = k >> 1, outer = k & 1;
        x = g.ax + (col - 1.5) * g.dx;
        y = g.by + g.dy * (outer ? 1.5 : 0.5);
        idx = (n + 2 + outer) * P + col;
    }
    const double prefac = g.dx * g.rhoinv * dt / (3 * M_PI);
    const double xm0 = x - g.ax, xp0 = x + g.ax, ysq = y * y;
    double su = 0, sv = 0;
    for (int jq = lane; jq < me; jq += 32) {
        double xms = xm0 - jq * g.dx, xps = xp0 + jq * g.dx, pp = gs.gp[jq];
        double rm = xms * xms + ysq;
        rm = 1 / (rm * rm);
        double fsu, fsv;
        if (g.x_sym) {
            double rp = xps * xps + ysq;
            rp = 1 / (rp * rp);
            fsu = pp * (xms * rm + xps * rp);
            fsv = -pp * ((xms * xms - ysq) * rm + (xps * xps - ysq) * rp);
        } else {
            fsu = pp * xms * rm;
            fsv = -pp * (xms * xms - ysq) * rm;
        }
        double w = (jq == 0 || jq == me - 1) ? 1. : ((jq & 1) ? 4. : 2.);
        su += w * fsu;
        sv += w * fsv;
    }
    for (int o = 16; o > 0; o >>= 1) {
        su += __shfl_down_sync(0xffffffffu, su, o);
        sv += __shfl_down_sync(0xffffffffu, sv, o);
    }
    if (lane == 0) {
        double un = f.u[idx] + 2 * y * prefac * su;
        double vn = f.v[idx] + prefac * sv;
        f.u[idx] = un;
        f.v[idx] = vn;
        if (right_row >= 0 && !g.x_sym) {
            // fluid_2d_sio.cc:271-276: mirror onto the left ghosts
            int j = right_row, outer = warp & 1;
            int li = (j + 2) * P + (outer ? 0 : 1);
            f.u[li] = -un;
            f.v[li] = vn;
        }
    }
}

// --------------------------------------------------- viscous boundaries
// fluid_2d_sio.cc:294-343 in one CTA (three dependent phases).
__global__ void k_viscous_bc(Grid g, Fields f, Gas gs) {
    const int m = g.m, n = g.n, P = m + 4, ml = m + 4;
    double* u = f.u;
    double* v = f.v;
    if (g.x_sym) {
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            int c = (j + 2) * P + 2;
            u[c - 1] = -u[c];
            v[c - 1] = v[c];
            u[c - 2] = -u[c + 1];
            v[c - 2] = v[c + 1];
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < ml; k += blockDim.x) {
        double un_edge = g.muinv * gs.tau[k];
        u[P + k] = u[2 * P + k] - g.dy * un_edge;
        u[k] = u[3 * P + k] - 3 * g.dy * un_edge;
    }
    __syncthreads();
    for (int k = 1 + threadIdx.x; k < m + 2; k += blockDim.x) {
        double uxa = 0.5 * g.xsp * (u[P + k + 1] - u[P + k - 1]);
        double uxb = 0.5 * g.xsp * (u[k + 1] - u[k - 1]);
        double v1 = v[2 * P + k] + g.dy * uxa;
        v[P + k] = v1;
        v[k] = v1 + g.dy * uxb;
    }
}

/** k_viscous_bc without its barriers, over many blocks: thread t < m+4
 * takes column t of the two bottom ghost rows, recomputing what the earlier
 * phases would have left in the cells it reads (the mirrored ghost columns
 * of rows 0 and 1, the u ghost rows at its neighbouring columns) by the same
 * expressions; the threads after them mirror the left ghost columns of the
 * rows. The values written are the single-CTA kernel's, bit for bit. */
__global__ void k_viscous_bc_par(Grid g, Fields f, Gas gs) {
    const int m = g.m, n = g.n, P = m + 4, ml = m + 4;
    double* u = f.u;
    double* v = f.v;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ml) {
        const int j = t - ml;
        if (!g.x_sym || j >= n) return;
        const int c = (j + 2) * P + 2;
        u[c - 1] = -u[c];
        v[c - 1] = v[c];
        u[c - 2] = -u[c + 1];
        v[c - 2] = v[c + 1];
        return;
    }
    // row r (0 or 1) of u at column k as the mirroring leaves it
    auto urow = [&](int r, int k) -> double {
        const int base = (2 + r) * P;
        return (g.x_sym && k < 2) ? -u[base + 3 - k] : u[base + k];
    };
    // the u ghost rows -1 (lo = false) and -2 (lo = true) at column k
    auto ughost = [&](int k, bool lo) -> double {
        double un_edge = g.muinv * gs.tau[k];
        return lo ? urow(1, k) - 3 * g.dy * un_edge : urow(0, k) - g.dy * un_edge;
    };
    const int k = t;
    u[P + k] = ughost(k, false);
    u[k] = ughost(k, true);
    if (k >= 1 && k < m + 2) {
        double uxa = 0.5 * g.xsp * (ughost(k + 1, false) - ughost(k - 1, false));
        double uxb = 0.5 * g.xsp * (ughost(k + 1, true) - ughost(k - 1, true));
        const double v0 = (g.x_sym && k < 2) ? v[2 * P + 3 - k] : v[2 * P + k];
        double v1 = v0 + g.dy * uxa;
        v[P + k] = v1;
        v[k] = v1 + g.dy * uxb;
    }
}

// ------------------------------------------------------- viscous sources
// fluid_2d.cc:279-324: right-hand sides of the u and v systems.
__global__ void k_visc_rhs(Grid g, Fields f, Gas gs, double vfx, double vfy, double* __restrict__ su,
                           double* __restrict__ sv) {
    CELL_LOOP
    const double* u = f.u;
    const double* v = f.v;
    double a = f.fc0[c], b = f.fc1[c];
    if (!g.x_sym && i == 0) {
        a += vfx * u[c - 1];
        b += vfx * v[c - 1];
    }
    if (i == g.m - 1) {
        a += vfx * u[c + 1];
        b += vfx * v[c + 1];
    }
    if (j == g.n - 1) {
        a += vfy * u[c + P];
        b += vfy * v[c + P];
    }
    if (j == 0) {
        double dudy = g.muinv * 0.5 * (gs.tau_old[i + 2] + gs.tau[i + 2]);
        a -= vfy * g.dy * dudy;
        double dvdy = -0.5 * g.xsp * (u[c + 1] - u[c - 1]);
        b -= vfy * g.dy * dvdy;
    }
    su[i + g.m * j] = a;
    sv[i + g.m * j] = b;
}

// ------------------------------------------------------------ FEM source
// fluid_2d.cc:337-377 on the (m+1) x (n+1) nodes; vel0/vel1 are the
// provisional velocities (the viscous solutions when implicit).
__global__ void k_fem_rhs(Grid g, Fields f, Gas gs, CellView c0v, CellView c1v, double dt, double a_cc_edge,
                          double a_cc_mid, double* __restrict__ src) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int m = g.m, n = g.n, me = m + 1, P = m + 4;
    if (i > m || j > n) return;
    if (j == 0) {
        // fluid_2d.cc:377 with mgs_fem::a_cc(i,i) (mgs_fem.hh:55-57)
        src[i] = ((i > 0 && i < m) ? a_cc_mid : a_cc_edge) * gs.gp[i];
        return;
    }
    double spx = 0, spy = 0;
    if (i != 0) {
        spx += c0v.at(i - 1, j - 1);
        spy += c1v.at(i - 1, j - 1);
    }
    if (i != 0 && j < n) {
        spx += c0v.at(i - 1, j);
        spy -= c1v.at(i - 1, j);
    }
    if (i != m) {
        spx -= c0v.at(i, j - 1);
        spy += c1v.at(i, j - 1);
    }
    if (i != m && j < n) {
        spx -= c0v.at(i, j);
        spy -= c1v.at(i, j);
    }
    double s = 0.5 * (g.dy * spx + g.dx * spy) * g.rho / dt;
    const double* u = f.u;
    const double* v = f.v;
    const double fl = 0.25 * g.dy * g.rho / dt;
    if (!g.x_sym && i == 0) {
        if (j < n) s += fl * (c0v.at(0, j) + u[(j + 2) * P + 1]);
        s += fl * (c0v.at(0, j - 1) + u[(j + 1) * P + 1]);
    }
    if (i == m) {
        if (j < n) s -= fl * (c0v.at(m - 1, j) + u[(j + 2) * P + m + 2]);
        s -= fl * (c0v.at(m - 1, j - 1) + u[(j + 1) * P + m + 2]);
    }
    if (j == n) {
        const double ft = 0.25 * g.dx * g.rho / dt;
        if (i > 0) s -= ft * (c1v.at(i - 1, n - 1) + v[(n + 2) * P + i + 1]);
        if (i < m) s -= ft * (c1v.at(i, n - 1) + v[(n + 2) * P + i + 2]);
    }
    src[i + me * j] = s;
}

// ------------------------------------------------------ velocity update
// fluid_2d.cc:383-396.
__global__ void k_vel_update(Grid g, Fields f, CellView c0v, CellView c1v, const double* __restrict__ z, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int m = g.m, n = g.n, me = m + 1, P = m + 4;
    if (i > m || j > n) return;
    int c = (j + 2) * P + i + 2;
    const double* sop = z + i + me * j;
    f.p[c] = *sop;
    if (i < m && j < n) {
        f.u[c] = c0v.at(i, j) - 0.5 * dt * g.rhoinv * g.xsp * (sop[me + 1] + sop[1] - sop[me] - *sop);
        f.v[c] = c1v.at(i, j) - 0.5 * dt * g.rhoinv * g.ysp * (sop[me + 1] - sop[1] + sop[me] - *sop);
    }
}

// ------------------------------------------------------------- tracers
// fluid_2d::update_tracers (fluid_2d.cc:507-526): each tracer moves by dt
// times the bilinear interpolation of the cell-centred velocity around it,
// the cell index clamped to [-1, m-1] x [-1, n-1] (ghost cells included).
__global__ void k_tracers(Grid g, const double* __restrict__ u, const double* __restrict__ v,
                          double* __restrict__ tm, int ntrace, double dt) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntrace) return;
    double* tp = tm + 2 * t;
    double x = (tp[0] - g.ax) * g.xsp - 0.5, y = (tp[1] - g.ay) * g.ysp - 0.5;
    int i = int(x);
    if (i < -1) i = -1;
    if (i > g.m - 1) i = g.m - 1;
    int j = int(y);
    if (j < -1) j = -1;
    if (j > g.n - 1) j = g.n - 1;
    x -= i;
    y -= j;
    const int P = g.m + 4, c = (j + 2) * P + i + 2;
    tp[0] += dt * ((1 - y) * (u[c] * (1 - x) + u[c + 1] * x) + y * (u[c + P] * (1 - x) + u[c + P + 1] * x));
    tp[1] += dt * ((1 - y) * (v[c] * (1 - x) + v[c + 1] * x) + y * (v[c + P] * (1 - x) + v[c + P + 1] * x));
}

// ------------------------------------------------- non-inertial frame
// fluid_2d::adjust_frame (fluid_2d_sio.cc:228-253): the frame velocity from
// the two rows around the liquid's bottom edge (row -1 and row 0), either a
// Lagrange interpolant at the centre (mode 1) or the mean over columns
// [a, b) summed in column order (mode 2); one thread, so the sum's order is
// the reference's.
__global__ void k_frame_velocity(Grid g, const double* __restrict__ v, int mode, int a, int b, double* vacc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int P = g.m + 4;
    const double* fm = v + 2 * P + 2;
    const double* fb = fm - P;
    double V;
    if (mode == 1) {
        const int m2 = g.m / 2;
        V = g.x_sym ? 0.5625 * (fb[0] + fm[0]) - 0.0625 * (fb[1] + fm[1])
                    : 0.28125 * (fb[m2 - 1] + fb[m2] + fm[m2 - 1] + fm[m2]) -
                          0.03125 * (fb[m2 - 2] + fb[m2 + 1] + fm[m2 - 2] + fm[m2 + 1]);
    } else {
        V = 0;
        for (int i = a; i < b; i++) V += fm[i] + fb[i];
        V *= 0.5 / (b - a);
    }
    *vacc = V;
}
/** Subtracts the frame velocity from v over the whole ghosted grid and from
 * the gas layer's Vframe. */
__global__ void k_frame_apply(double* __restrict__ v, long tot, const double* __restrict__ vacc, double* vframe) {
    const double V = *vacc;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < tot; k += long(gridDim.x) * blockDim.x) v[k] -= V;
    if (blockIdx.x == 0 && threadIdx.x == 0) *vframe -= V;
}

// ------------------------------------------------ multigrid initial guess
// mgs_common::initial_guess (mgs_common.cc:17-50). The decision is made from
// device-resident times so that a captured graph replays it correctly. One
// launch: thread 0 of every block copies the history to shared memory, and
// the last block to arrive (an atomic count in the history itself) advances
// the history, after every block has read the old one.
//
// QUAD adds a second-order variant: with three past solutions z (at t0),
// zprev (t_prev) and zprev2 (t_prev2) the guess is the quadratic Lagrange
// extrapolation to t; with two it is the linear rule. This changes only the
// starting iterate of the solve, not its converged result.
//
// The target time is *d_time + tadd: a guess enqueued before the kernel that
// advances the clock by dt/2 passes tadd = dt/2 and gets the same double that
// the clock will hold (the same single rounded addition).
/** Points per thread of k_guess. */
static constexpr int GUESS_PER = 3;

template <bool QUAD>
__global__ void __launch_bounds__(256, 4) k_guess(double* __restrict__ z, double* __restrict__ zprev,
                                                  double* __restrict__ zprev2, int n, GuessHist* h,
                                                  const double* d_time, double tadd, int* err) {
    __shared__ double s_t[4];   // t, t0, t_prev, t_prev2
    __shared__ double s_w[3];   // the extrapolation's weights (their meaning by rule below)
    __shared__ int s_sc, s_head;
    // each thread takes GUESS_PER points, a grid-size apart; their values
    // are loaded before the history header is, so the two overlap
    const int k0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    double vz[GUESS_PER], va[GUESS_PER], vb[GUESS_PER];
#pragma unroll
    for (int u = 0; u < GUESS_PER; u++) {
        const int k = k0 + u * stride;
        const bool in = k < n;
        vz[u] = in ? z[k] : 0.;
        va[u] = in ? zprev[k] : 0.;
        vb[u] = (QUAD && in) ? zprev2[k] : 0.;
    }
    if (threadIdx.x == 0) {
        s_t[0] = *d_time + tadd;
        s_t[1] = h->t0;
        s_t[2] = h->t_prev;
        s_t[3] = h->t_prev2;
        s_sc = h->scount;
        s_head = h->head;
    }
    __syncthreads();
    {
        // the extrapolation weights, once per block: thread q < 3 forms
        // weight q (linear: z = w0 zz - w1 v1 with w0, w1 over one
        // reciprocal; quadratic: the Lagrange weights, z = w0 zz + w1 v1 +
        // w2 v2)
        const double t = s_t[0], t0 = s_t[1], t1 = s_t[2], t2 = s_t[3];
        const int q = threadIdx.x;
        if (q < 3) s_w[q] = 0.;
        if (q < 3 && s_sc >= 2 && !(fabs(t0 - t1) < 2.220446049250313e-16 * 10)) {
            if (!QUAD || s_sc == 2) {
                double a = 1. / (t0 - t1);
                s_w[q] = q == 0 ? (t - t1) * a : (q == 1 ? (t - t0) * a : 0.);
            } else {
                const double tq = q == 0 ? t0 : (q == 1 ? t1 : t2);
                const double ta = q == 0 ? t1 : t0, tb = q == 2 ? t1 : t2;
                s_w[q] = (t - ta) * (t - tb) / ((tq - ta) * (tq - tb));
            }
        }
    }
    __syncthreads();
    const int sc = s_sc;
    const double t = s_t[0], t0 = s_t[1], t1 = s_t[2];
    const bool dup = fabs(t0 - t1) < 2.220446049250313e-16 * 10;
    const bool lin = !QUAD || sc == 2;
    const double w0 = s_w[0], w1 = s_w[1], w2 = s_w[2];
    // quadratic history: h1 holds the solution at t_prev, h2 the one at
    // t_prev2; the newest history replaces h2's and the two swap roles
    const bool swap = QUAD && s_head;
    double* h1 = swap ? zprev2 : zprev;
    double* h2 = swap ? zprev : zprev2;
#pragma unroll
    for (int u = 0; u < GUESS_PER; u++) {
        const int k = k0 + u * stride;
        if (k >= n) continue;
        const double v1 = swap ? vb[u] : va[u], v2 = swap ? va[u] : vb[u];
        if (sc < 2) {
            if (sc == 1) h1[k] = vz[u];
        } else if (!dup) {
            double zz = vz[u];
            if (lin) z[k] = w0 * zz - w1 * v1;
            else z[k] = w0 * zz + w1 * v1 + w2 * v2;
            if (QUAD) h2[k] = zz;
            else h1[k] = zz;
        }
    }
    if (threadIdx.x != 0) return;
    __threadfence();
    if (atomicAdd(&h->arrive, 1u) != gridDim.x - 1) return;
    __threadfence();
    h->arrive = 0;
    if (sc < 2) {
        if (sc == 1) h->t0 = t;
        else h->t_prev = t;
        h->scount = sc + 1;
    } else if (dup) {
        atomicOr(err, DEV_DUP_TIME);
    } else {
        if (QUAD) {
            h->t_prev2 = t1;
            h->head = s_head ^ 1;
        }
        h->t_prev = t0;
        h->t0 = t;
        if (QUAD && sc < 3) h->scount = sc + 1;
    }
}

// --------------------------------------------------------------- launch
static dim3 cell_block(const Grid& g) {
    return g.blk_x > 0 ? dim3(g.blk_x, g.blk_y) : dim3(32, 8);
}
static dim3 cell_grid(const Grid& g, int extra = 0) {
    dim3 b = cell_block(g);
    return dim3((g.m + extra + b.x - 1) / b.x, (g.n + extra + b.y - 1) / b.y);
}

int launch_stage1(cudaStream_t s, const Grid& g, const Fields& f, double dt) {
    k_stage1<<<cell_grid(g), cell_block(g), 0, s>>>(g, f, dt);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_stage2(cudaStream_t s, const Grid& g, const Fields& f) {
    k_stage2<<<cell_grid(g), cell_block(g), 0, s>>>(g, f);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_stage34(cudaStream_t s, const Grid& g, const Fields& f, double dt) {
    k_stage34<<<cell_grid(g), cell_block(g), 0, s>>>(g, f, dt);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_stage5_src(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs, double dt, double* src) {
    k_stage5_src<<<cell_grid(g), cell_block(g), 0, s>>>(g, f, gs, dt, src);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_advect(cudaStream_t s, const Grid& g, const Fields& f, double dt, double* src) {
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_advect, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ADV_SMEM)) != cudaSuccess)
            return VDI_ERR_CUDA;
        attr = true;
    }
    dim3 grid((g.m + ADV_TX - 1) / ADV_TX, (g.n + ADV_TY - 1) / ADV_TY);
    k_advect<<<grid, ADV_NT, ADV_SMEM, s>>>(g, f, dt, src);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_mac_src_bottom(cudaStream_t s, const Grid& g, const Gas& gs, double dt, double* src) {
    k_mac_src_bottom<<<(g.m + 255) / 256, 256, 0, s>>>(g, gs, dt, src);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_mac_advect(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs, const double* q, double dt,
                      double* d_time) {
    k_mac_advect<<<cell_grid(g), cell_block(g), 0, s>>>(g, f, gs, q, dt, d_time);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_inviscid_bc(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs, double dt) {
    long warps = 2L * g.n + 2L * (g.m + 4);
    k_inviscid_bc<<<int((warps * 32 + 255) / 256), 256, 0, s>>>(g, f, gs, dt);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_viscous_bc(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs) {
    const char* e = getenv("VDI_VISC_BC_PAR");
    if (e && atoi(e) == 0) {
        k_viscous_bc<<<1, 1024, 0, s>>>(g, f, gs);
    } else {
        const int threads = (g.m + 4) + (g.x_sym ? g.n : 0);
        k_viscous_bc_par<<<(threads + 255) / 256, 256, 0, s>>>(g, f, gs);
    }
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_visc_rhs(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs, double vfx, double vfy,
                    double* su, double* sv) {
    k_visc_rhs<<<cell_grid(g), cell_block(g), 0, s>>>(g, f, gs, vfx, vfy, su, sv);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_fem_rhs(cudaStream_t s, const Grid& g, const Fields& f, const Gas& gs, CellView c0, CellView c1, double dt,
                   double a_cc_edge, double a_cc_mid, double* src) {
    k_fem_rhs<<<cell_grid(g, 1), cell_block(g), 0, s>>>(g, f, gs, c0, c1, dt, a_cc_edge, a_cc_mid, src);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_vel_update(cudaStream_t s, const Grid& g, const Fields& f, CellView c0, CellView c1, const double* z,
                      double dt) {
    k_vel_update<<<cell_grid(g, 1), cell_block(g), 0, s>>>(g, f, c0, c1, z, dt);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_tracers(cudaStream_t s, const Grid& g, const Fields& f, double* tm, int ntrace, double dt) {
    if (ntrace <= 0) return VDI_OK;
    k_tracers<<<(ntrace + 127) / 128, 128, 0, s>>>(g, f.u, f.v, tm, ntrace, dt);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}
int launch_frame(cudaStream_t s, const Grid& g, const Fields& f, int mode, int a, int b, double* vacc,
                 double* vframe) {
    const long tot = long(g.m + 4) * (g.n + 4);
    k_frame_velocity<<<1, 32, 0, s>>>(g, f.v, mode, a, b, vacc);
    k_frame_apply<<<int(std::min<long>((tot + 255) / 256, 1184)), 256, 0, s>>>(f.v, tot, vacc, vframe);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}

int launch_guess(cudaStream_t s, double* z, double* zprev, double* zprev2, int n, GuessHist* h,
                 const double* d_time, double tadd, int quadratic, int* err) {
    if (n <= 0) return VDI_OK;
    if (quadratic)
        k_guess<true><<<(n + 256 * GUESS_PER - 1) / (256 * GUESS_PER), 256, 0, s>>>(z, zprev, zprev2, n, h, d_time,
                                                                                     tadd, err);
    else
        k_guess<false><<<(n + 256 * GUESS_PER - 1) / (256 * GUESS_PER), 256, 0, s>>>(z, zprev, zprev2, n, h, d_time,
                                                                                      tadd, err);
    return cudaGetLastError() == cudaSuccess ? VDI_OK : VDI_ERR_CUDA;
}

}  // namespace vdi
