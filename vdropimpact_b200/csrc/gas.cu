// Gas layer (gas_layer.cc, gas_layer_solve.cc) and the tridiagonal solver
// (tri_solve.cc) as single-CTA kernels. The whole update — height advection,
// the Newton loop with one tridiagonal solve per step, and the liquid
// pressure and shear stress — runs inside one launch, so the step needs no
// host round trip and the launch can overlap the liquid's advection kernels.
//
// Tridiagonal systems are solved by cyclic reduction in shared memory when
// every row is diagonally dominant, and otherwise by Gaussian elimination
// with partial pivoting (the algorithm of LAPACK dgtsv, which the reference
// calls at tri_solve.cc:28) on one thread.
//
// update_height (gas_layer_solve.cc:133-162) updates h[i] in place, so the
// reference's loop is a recurrence: iteration i reads the new h[i-1], h[i-2].
// The kernel evaluates it as a fixed-point iteration, H_{k+1}[i] =
// F_i(H_k[0..i-1], h_old[i..]), for all i at once; once an iteration changes
// no bit, every entry satisfies the recurrence and equals the sequential
// result exactly. A cap on the iterations falls back to the sequential loop.
//
// Compiled with -fmad=false: the arithmetic follows the reference's
// expression order.
#include "step_kernels.hh"

#include <cmath>

namespace vdi {

static constexpr int GAS_THREADS = 1024;
static constexpr int FP_MAX_ITERS = 256;
// gas_layer_solve.hh:11-18
static constexpr double PRESSURE_R_ERROR = 2.220446049250313e-16 * 1e8;
static constexpr double NEWTON_THRESH = PRESSURE_R_ERROR * PRESSURE_R_ERROR;
static constexpr int MAX_NEWTON_STEPS = 256;

__device__ __forceinline__ double gwarp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

/** Block sum, valid in every thread (deterministic for a fixed block size). */
__device__ double gblock_sum(double v, double* ws) {
    v = gwarp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) ws[w] = v;
    __syncthreads();
    if (w == 0) {
        double r = lane < int(blockDim.x >> 5) ? ws[lane] : 0.;
        r = gwarp_sum(r);
        if (lane == 0) ws[32] = r;
    }
    __syncthreads();
    return ws[32];
}

__host__ __device__ static inline int pad_pow2m1(int n) {
    int p = 1;
    while (p - 1 < n) p <<= 1;
    return p - 1;
}

/** Solves the n-row system held in a, b, c, d (length >= Np, rows n..Np-1
 * free for padding) by cyclic reduction; solution in x. Requires a[0] and
 * c[n-1] to be zero. Called by the whole block. */
__device__ void cyclic_reduction(int n, int Np, double* a, double* b, double* c, double* d, double* x) {
    for (int k = n + threadIdx.x; k < Np; k += blockDim.x) {
        a[k] = 0; b[k] = 1; c[k] = 0; d[k] = 0;
    }
    __syncthreads();
    int half = (Np + 1) >> 1;
    for (int s = 1; s < half; s <<= 1) {
        for (int i = 2 * s - 1 + 2 * s * threadIdx.x; i < Np; i += 2 * s * blockDim.x) {
            int il = i - s, ir = i + s;
            double k1 = a[i] / b[il];
            double k2 = ir < Np ? c[i] / b[ir] : 0.;
            double ai = -a[il] * k1;
            double ci = ir < Np ? -c[ir] * k2 : 0.;
            double bi = b[i] - c[il] * k1 - (ir < Np ? a[ir] * k2 : 0.);
            double di = d[i] - d[il] * k1 - (ir < Np ? d[ir] * k2 : 0.);
            a[i] = ai; b[i] = bi; c[i] = ci; d[i] = di;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        int mid = (Np - 1) >> 1;
        x[mid] = d[mid] / b[mid];
    }
    __syncthreads();
    for (int s = half >> 1; s >= 1; s >>= 1) {
        for (int i = s - 1 + 2 * s * threadIdx.x; i < Np; i += 2 * s * blockDim.x) {
            double xl = i - s >= 0 ? x[i - s] : 0.;
            double xr = i + s < Np ? x[i + s] : 0.;
            x[i] = (d[i] - a[i] * xl - c[i] * xr) / b[i];
        }
        __syncthreads();
    }
}

/** Gaussian elimination with partial pivoting on one thread (the algorithm
 * of LAPACK dgtsv). dl = a+1, du = c, du2 scratch of n entries. Returns
 * info (0 ok, k>0: zero pivot at row k). Solution in d. */
__device__ int gepp_tridiag(int n, double* a, double* b, double* c, double* d, double* du2) {
    double* dl = a + 1;
    for (int i = 0; i < n - 1; i++) {
        if (fabs(b[i]) >= fabs(dl[i])) {
            if (b[i] == 0) return i + 1;
            double fact = dl[i] / b[i];
            b[i + 1] -= fact * c[i];
            d[i + 1] -= fact * d[i];
            if (i < n - 2) du2[i] = 0;
        } else {
            double fact = b[i] / dl[i];
            b[i] = dl[i];
            double temp = b[i + 1];
            b[i + 1] = c[i] - fact * temp;
            if (i < n - 2) {
                du2[i] = c[i + 1];
                c[i + 1] = -fact * du2[i];
            }
            c[i] = temp;
            temp = d[i];
            d[i] = d[i + 1];
            d[i + 1] = temp - fact * d[i + 1];
        }
    }
    if (b[n - 1] == 0) return n;
    d[n - 1] /= b[n - 1];
    if (n > 1) d[n - 2] = (d[n - 2] - c[n - 2] * d[n - 1]) / b[n - 2];
    for (int i = n - 3; i >= 0; i--) d[i] = (d[i] - c[i] * d[i + 1] - du2[i] * d[i + 2]) / b[i];
    return 0;
}

/** Solves the system in place (solution in d). Whole block. Returns info
 * in every thread; *pivoted set when the fallback ran. */
__device__ int tri_solve_block(int n, int Np, double* a, double* b, double* c, double* d, double* x,
                               double* ws, int* pivoted) {
    __shared__ int info_s;
    if (threadIdx.x == 0) {
        a[0] = 0;
        c[n - 1] = 0;
    }
    __syncthreads();
    int bad = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (!(fabs(b[i]) >= fabs(a[i]) + fabs(c[i])) || b[i] == 0) bad = 1;
    bad = __syncthreads_or(bad);
    if (!bad) {
        cyclic_reduction(n, Np, a, b, c, d, x);
        for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = x[i];
        __syncthreads();
        *pivoted = 0;
        return 0;
    }
    if (threadIdx.x == 0) info_s = gepp_tridiag(n, a, b, c, d, x);
    __syncthreads();
    *pivoted = 1;
    return info_s;
}

/** One CTA solves the whole system in shared memory (launch_tri_solve
 * rejects systems that do not fit). */
__global__ void k_tri_solve(int n, int Np, double* ga, double* gb, double* gc, double* gd, int* out_pivoted) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double ws[33];
    double* a = sm;
    double* b = a + Np;
    double* c = b + Np;
    double* d = c + Np;
    double* x = d + Np;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a[i] = ga[i]; b[i] = gb[i]; c[i] = gc[i]; d[i] = gd[i];
    }
    __syncthreads();
    int piv = 0;
    int info = tri_solve_block(n, Np, a, b, c, d, x, ws, &piv);
    for (int i = threadIdx.x; i < n; i += blockDim.x) gd[i] = d[i];
    if (threadIdx.x == 0 && out_pivoted) out_pivoted[0] = info != 0 ? -info : piv;
}

// ----------------------------------------------------------------- gas
struct HCtx {
    int m, x_sym;
    const double* H;    // current iterate (new values for indices < i)
    const double* Ho;   // values at the start of the update
};

__device__ __forceinline__ double hv(const HCtx& h, int k, int i) { return k < i ? h.H[k] : h.Ho[k]; }

// gas_layer_solve.cc:173-177 evaluated as at iteration i of the loop
__device__ __forceinline__ double h_ref(const HCtx& h, int k, int i) {
    const int m = h.m;
    if (k >= 0) {
        if (k < m) return hv(h, k, i);
        return k == m ? 2 * hv(h, m - 1, i) - hv(h, m - 2, i) : 3 * hv(h, m - 1, i) - 2 * hv(h, m - 2, i);
    }
    if (h.x_sym) return k == -1 ? hv(h, 0, i) : hv(h, 1, i);
    return k == -1 ? 2 * hv(h, 0, i) - hv(h, 1, i) : 3 * hv(h, 0, i) - 2 * hv(h, 1, i);
}

// gas_layer_solve.cc:165-167
__device__ __forceinline__ double eno2(double p0, double p1, double p2, double p3) {
    return fabs(p0 - 2 * p1 + p2) > fabs(p1 - 2 * p2 + p3) ? 3 * p1 - 4 * p2 + p3 : p0 - p2;
}

/** ht at iteration i of update_height (gas_layer_solve.cc:136-148). */
__device__ __forceinline__ double height_rate(const HCtx& h, int i, double uc, double vc, double Vframe) {
    double hi = h.Ho[i];
    double dhdx = uc > 0 ? eno2(h_ref(h, i + 1, i), hi, h_ref(h, i - 1, i), h_ref(h, i - 2, i))
                         : -eno2(h_ref(h, i - 1, i), hi, h_ref(h, i + 1, i), h_ref(h, i + 2, i));
    return -uc * dhdx + vc - Vframe;
}

/** calculate_liquid_fields (gas_layer_solve.cc:229-249). Whole block. */
__device__ void liquid_fields(const GasPrm& P, const Gas& g) {
    const int m = P.m;
    const double fac = 0.5 * P.sigma * P.xxsp, fac2 = P.sigma / P.R;
    const double* h = g.h;
    const double* pg = g.pg;
    double* p = g.gp;
    for (int i = threadIdx.x; i <= m; i += blockDim.x) {
        double val;
        if (i == 0) val = P.x_sym ? pg[0] + 2 * fac * (h[1] - h[0]) - fac2 : pg[0];
        else if (i == 1) val = P.x_sym ? pg[1] + fac * (h[2] - h[1]) - fac2 : pg[1];
        else if (i < m - 1) val = pg[i] + fac * (h[i + 1] - h[i] - h[i - 1] + h[i - 2]) - fac2;
        else val = pg[i];
        p[i] = val;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) g.tau[i] = -0.5 * P.xsp * P.mu * (p[i + 1] - p[i]) * h[i];
    __syncthreads();
}

/** calculate_hx (gas_layer_solve.cc:55-59). Whole block. */
__device__ void calc_hx(const GasPrm& P, const Gas& g) {
    const int m = P.m;
    for (int i = 1 + threadIdx.x; i < m; i += blockDim.x) g.hx[i] = P.xsp * (g.h[i] - g.h[i - 1]);
    __syncthreads();
    if (threadIdx.x == 0) {
        g.hx[0] = P.x_sym ? 0 : g.hx[1];
        g.hx[m] = g.hx[m - 1];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(GAS_THREADS)
k_gas_update(GasPrm P, Gas g, const double* __restrict__ u, const double* __restrict__ v, int pitch,
             const double* d_vframe, double dt, double* d_time, double* gwork, int use_smem, int* err,
             GasStats* stats) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double ws[33];
    const int m = P.m, me = m + 1, ml = m + 4;
    const int Np = pad_pow2m1(me);
    double* W = use_smem ? sm : gwork;
    const double Vframe = *d_vframe;

    // gas_layer::update: keep the previous pressure and shear stress
    for (int i = threadIdx.x; i < me; i += blockDim.x) g.gp_old[i] = g.gp[i];
    for (int i = threadIdx.x; i < ml; i += blockDim.x) g.tau_old[i] = g.tau[i];

    // ---------------------------------------------------- update_height
    double* UC = W;
    double* VC = UC + m;
    double* HO = VC + m;
    double* HA = HO + m;
    double* HB = HA + m;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        int c0 = 2 * pitch + i + 2, cb = pitch + i + 2;   // rows j = 0 and j = -1
        UC[i] = 0.25 * P.xsp * (u[c0] + u[cb]);
        VC[i] = 0.5 * (v[c0] + v[cb]);
        HO[i] = g.h[i];
        HA[i] = g.h[i];
    }
    __syncthreads();
    int iters = 0;
    bool converged = false;
    while (iters < FP_MAX_ITERS) {
        HCtx hc{m, P.x_sym, HA, HO};
        int changed = 0;
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            double ht = height_rate(hc, i, UC[i], VC[i], Vframe);
            double hn = HO[i] + dt * ht;
            HB[i] = hn;
            if (!(hn == HA[i])) changed = 1;
        }
        iters++;
        changed = __syncthreads_or(changed);
        double* t = HA; HA = HB; HB = t;
        if (!changed) {
            converged = true;
            break;
        }
    }
    if (!converged) {
        // sequential evaluation of the reference loop
        if (threadIdx.x == 0) {
            for (int i = 0; i < m; i++) HA[i] = HO[i];
            for (int i = 0; i < m; i++) {
                HCtx hc{m, P.x_sym, HA, HO};
                double ht = height_rate(hc, i, UC[i], VC[i], Vframe);
                HA[i] = HO[i] + dt * ht;
            }
        }
        __syncthreads();
    }
    {
        HCtx hc{m, P.x_sym, HA, HO};
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            double ht = height_rate(hc, i, UC[i], VC[i], Vframe);
            g.ht[i] = ht;
            g.h[i] = HO[i] + dt * ht;
            g.fbd[i] += dt * VC[i];
        }
    }
    __syncthreads();
    calc_hx(P, g);

    // ------------------------------------------------- Newton iteration
    for (int i = threadIdx.x; i < me; i += blockDim.x) g.pg_old[i] = g.pg[i];
    __syncthreads();
    double* A = W;
    double* B = A + Np;
    double* C = B + Np;
    double* D = C + Np;
    double* X = D + Np;
    const double dtinv = 1. / dt;
    const double xsp = P.xsp, xxsp = P.xxsp, mu = P.mu, alpha = P.alpha, Pamb = P.Pamb;
    const double* h = g.h;
    const double* ht = g.ht;
    const double* hx = g.hx;
    double* pg = g.pg;
    const double* pg_old = g.pg_old;
    int nstep = 0, naccept = 0, failed = 0, npiv = 0;
    const int i0 = P.x_sym ? 0 : 1;
    do {
        if (++nstep > MAX_NEWTON_STEPS) {
            failed = DEV_NEWTON;
            break;
        }
        // gas_layer_solve.cc:67-126
        double part = 0;
        for (int i = threadIdx.x; i < me; i += blockDim.x) {
            double ai, bi, ci, di;
            if (i == me - 1) {
                ai = 0; bi = 1; ci = 0; di = -pg[me - 1];
            } else if (i < i0) {
                ai = 0; bi = 1; ci = 0; di = -pg[0];
            } else {
                double h_ns = i > 0 ? 0.5 * (h[i - 1] + h[i]) : h[i];
                double ht_ns = i > 0 ? 0.5 * (ht[i - 1] + ht[i]) : ht[i];
                double px = i > 0 ? 0.5 * xsp * (pg[i + 1] - pg[i - 1]) : 0;
                double pxx = i > 0 ? xxsp * (pg[i + 1] - 2 * pg[i] + pg[i - 1]) : xxsp * (pg[i + 1] - 2 * pg[i] + pg[i + 1]);
                double hsq = h_ns * h_ns;
                double hcu = hsq * h_ns;
                double br = 3 * hsq * hx[i] * px + hcu * pxx - 12 * mu * alpha * h_ns * dtinv - 12 * mu * ht_ns;
                ai = -xsp * alpha * hcu * px + pg[i] * (-1.5 * xsp * hsq * hx[i] + hcu * xxsp) +
                     Pamb * (-1.5 * xsp * hsq * hx[i] + hcu * xxsp);
                bi = br - 2 * pg[i] * hcu * xxsp - 2 * Pamb * hcu * xxsp;
                ci = xsp * alpha * hcu * px + pg[i] * (1.5 * xsp * hsq * hx[i] + hcu * xxsp) +
                     Pamb * (1.5 * xsp * hsq * hx[i] + hcu * xxsp);
                if (i == 0) ci += ai;
                di = -(12 * mu * alpha * h_ns * dtinv * pg_old[i] + alpha * hcu * px * px + pg[i] * br +
                       Pamb * (-12 * mu * ht_ns + 3 * hsq * hx[i] * px + hcu * pxx));
                part += di * di;
            }
            A[i] = ai; B[i] = bi; C[i] = ci; D[i] = di;
        }
        double ressq = gblock_sum(part, ws);
        int piv = 0;
        int info = tri_solve_block(me, Np, A, B, C, D, X, ws, &piv);
        npiv += piv;
        if (info != 0) {
            failed = DEV_TRI_SINGULAR;
            break;
        }
        for (int i = threadIdx.x; i < me; i += blockDim.x) pg[i] += D[i];
        __syncthreads();
        double res = ressq / me;
        if (!isfinite(res)) {
            failed = DEV_NONFINITE;
            break;
        }
        if (res < NEWTON_THRESH) naccept++;
        else naccept = 0;
    } while (naccept < 2);
    __syncthreads();

    liquid_fields(P, g);
    if (threadIdx.x == 0) {
        // gas_layer::apply_tau_bc (gas_layer.cc:25-30)
        double* t = g.tau;
        t[0] = -t[3];
        t[1] = -t[2];
        t[ml - 2] = -t[ml - 3];
        t[ml - 1] = -t[ml - 4];
        *d_time += 0.5 * dt;
        if (failed) atomicOr(err, failed);
        stats->updates += 1;
        stats->newton_steps += nstep;
        stats->pivot_fallbacks += npiv;
        stats->fixed_point_iters += iters;
        if (!converged) stats->sequential_fallbacks += 1;
    }
}

__global__ void k_gas_init(GasPrm P, Gas g, double h0, double V) {
    const int m = P.m;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        g.fbd[i] = 0;
        double x = P.ax + (i + 0.5) * P.dx;
        g.h[i] = h0 + 0.5 / P.R * x * x;
        g.ht[i] = -V;
    }
    for (int i = threadIdx.x; i <= m; i += blockDim.x) g.pg[i] = 0;
    __syncthreads();
    calc_hx(P, g);
    liquid_fields(P, g);
}

size_t gas_work_doubles(int m) {
    int Np = pad_pow2m1(m + 1);
    size_t a = 5 * size_t(m), b = 5 * size_t(Np);
    return a > b ? a : b;
}

static size_t gas_smem_limit() { return 220 * 1024; }

int launch_gas_update(cudaStream_t s, const GasPrm& gp, const Gas& gs, const double* u, const double* v, int pitch,
                      const double* d_vframe, double dt, double* d_time, double* work, int* err, GasStats* stats) {
    size_t bytes = gas_work_doubles(gp.m) * sizeof(double);
    int use_smem = bytes <= gas_smem_limit();
    static bool attr_set = false;
    if (!attr_set) {
        VDI_CUDA(cudaFuncSetAttribute(k_gas_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(gas_smem_limit())));
        attr_set = true;
    }
    k_gas_update<<<1, GAS_THREADS, use_smem ? bytes : 0, s>>>(gp, gs, u, v, pitch, d_vframe, dt, d_time, work,
                                                              use_smem, err, stats);
    VDI_CUDA(cudaGetLastError());
    return VDI_OK;
}

int launch_gas_init(cudaStream_t s, const GasPrm& gp, const Gas& gs, double h0, double V) {
    k_gas_init<<<1, GAS_THREADS, 0, s>>>(gp, gs, h0, V);
    VDI_CUDA(cudaGetLastError());
    return VDI_OK;
}

int launch_tri_solve(cudaStream_t s, int n, double* a, double* b, double* c, double* d, int* d_pivoted) {
    int Np = pad_pow2m1(n);
    size_t bytes = 5 * size_t(Np) * sizeof(double);
    if (bytes > gas_smem_limit()) {
        set_error("tri_solve: n=%d exceeds the shared-memory solver", n);
        return VDI_ERR_UNSUPPORTED_SIZE;
    }
    static bool attr_set = false;
    if (!attr_set) {
        VDI_CUDA(cudaFuncSetAttribute(k_tri_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(gas_smem_limit())));
        attr_set = true;
    }
    k_tri_solve<<<1, GAS_THREADS, bytes, s>>>(n, Np, a, b, c, d, d_pivoted);
    VDI_CUDA(cudaGetLastError());
    return VDI_OK;
}

}  // namespace vdi
