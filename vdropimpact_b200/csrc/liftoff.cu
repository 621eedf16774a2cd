// Lift-off search on the device: the reference's analysis tool
// (tt_analysis.cc:97-171) applied to the gas-layer height after every
// timestep (or every k-th), inside the step's CUDA graph.
//
// One CTA analyses one profile, the float32 values that the reference's frame
// output would hold (gas_layer_solve.cc:258-282):
//   - Gaussian smoothing with the tool's float32 accumulator
//     (tt_analysis.cc:36-57); the weights come from the host, where exp() is
//     the C library's, as in the tool;
//   - the minimum over the grid values and the interior minima of the
//     piecewise cubic Hermite interpolant (tt_analysis.cc:114-146), as a
//     parallel reduction that keeps the tool's sequential tie-break (the
//     first candidate, in the tool's visiting order, that attains the
//     minimum);
//   - the search update (tt_analysis.cc:148-163) by one thread.
// This file is compiled without FMA contraction so that every expression
// rounds as the tool's does; the tool reads q[m], one past the smoothed
// profile, in the tangent of its last interval (tt_analysis.cc:119) and this
// kernel reads 0 there.
#include "vdi_internal.hh"
#include "liftoff.hh"

#include <cfloat>
#include <cmath>
#include <vector>

namespace vdi {

namespace {

constexpr int LO_THREADS = 1024;

struct Cand {
    double v;      // height
    long seq;      // visiting order in the tool's loop (-1 for its initial value)
    double x;      // position
};

__device__ __forceinline__ bool better(const Cand& a, const Cand& b) {
    return a.v < b.v || (a.v == b.v && a.seq < b.seq);
}

__device__ __forceinline__ double hermite(double x, double t0, double t1, double t2, double t3) {
    return t0 * x * x * (3 - 2 * x) + x * (1 - x) * (-t1 * (1 - x) + t2 * x) + t3 * (2 * x * x * x - 3 * x * x + 1);
}

/** (xmin, fmin) of the profile h[0..m) into out; shared memory holds the
 * widened float32 profile, its smoothed copy and the positions. */
__device__ void profile_min_block(const double* __restrict__ h, const LiftoffCfg& c, double* sm, double* out) {
    const int m = c.m, tid = threadIdx.x;
    double* fs = sm;              // [m]   float32 heights
    double* q = fs + m;           // [m+1] smoothed (or raw) profile, q[m] = 0
    double* xs = q + m + 1;       // [m]   float32 positions
    for (int i = tid; i < m; i += blockDim.x) {
        fs[i] = double(float(h[i]));
        xs[i] = double(float(c.ax + (i + 0.5) * c.dx));
    }
    __syncthreads();
    const bool smoothed = c.mode == VDI_LIFTOFF_SMOOTHED;
    for (int i = tid; i < m; i += blockDim.x) {
        if (smoothed) {
            float v = 0.f;
            for (int off = -c.cut; off <= c.cut; off++) {
                int j = i + off;
                j = j < 0 ? -1 - j : (j >= m ? 2 * m - 1 - j : j);
                v = float(double(v) + c.w[off + c.cut] * fs[j]);
            }
            q[i] = double(v);
        } else {
            q[i] = fs[i];
        }
    }
    if (tid == 0) q[m] = 0.;
    __syncthreads();
    Cand best{fs[0], -1, xs[0]};
    for (int k = tid; k < m - 1; k += blockDim.x) {
        const double* f = q + k;
        const double t0 = f[1], t1 = 0.5 * (f[2] - *f), t2 = k == 0 ? (f[1] - *f) : 0.5 * (f[1] - f[-1]), t3 = *f;
        const double a = 6 * (t3 - t0) + 3 * (t1 + t2), b = 6 * t0 - 2 * t1 - 4 * t2 - 6 * t3, cc = t2;
        double det = b * b - 4 * a * cc;
        Cand g{f[1], 3L * k, xs[k + 1]};
        if (better(g, best)) best = g;
        if (smoothed && det >= 0) {
            det = sqrt(det);
            double xp = 0.5 * (-b + det), xm = 0.5 * (-b - det);
            if (0 < xp && xp < a) {
                xp /= a;
                Cand p{hermite(xp, t0, t1, t2, t3), 3L * k + 1, (1 - xp) * xs[k] + xp * xs[k + 1]};
                if (better(p, best)) best = p;
            }
            if (0 < xm && xm < a) {
                xm /= a;
                Cand p{hermite(xm, t0, t1, t2, t3), 3L * k + 2, (1 - xm) * xs[k] + xm * xs[k + 1]};
                if (better(p, best)) best = p;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        Cand r{__shfl_down_sync(0xffffffffu, best.v, o), __shfl_down_sync(0xffffffffu, best.seq, o),
               __shfl_down_sync(0xffffffffu, best.x, o)};
        if (better(r, best)) best = r;
    }
    __shared__ Cand wbest[LO_THREADS / 32];
    if ((tid & 31) == 0) wbest[tid >> 5] = best;
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < int(blockDim.x >> 5); w++)
            if (better(wbest[w], best)) best = wbest[w];
        out[0] = best.x;
        out[1] = best.v;
    }
}

/** One search step: analyses the profile when the step counter is a
 * multiple of c.every (tt_analysis.cc:148-163). */
__global__ void __launch_bounds__(LO_THREADS) k_liftoff(const double* __restrict__ h, LiftoffCfg c,
                                                        LiftoffState* st, double2* hist, long cap, double dt) {
    extern __shared__ double lsm[];
    __shared__ long s_n;
    __shared__ double res[2];
    if (threadIdx.x == 0) {
        s_n = st->counter;
        st->counter = s_n + 1;
    }
    __syncthreads();
    if (s_n % c.every) return;
    profile_min_block(h, c, lsm, res);
    if (threadIdx.x != 0) return;
    const double xmin = res[0], fmin = res[1];
    const long i = st->count;
    const double interval = dt * c.every;
    if (st->hsearch && fmin < st->gfmin) {
        st->gfmin = fmin;
        st->gimin = i;
        st->gxmin = xmin;
        if (st->efield && fmin < c.h_ev) {
            st->tmin0_ev = i * interval - xmin * xmin / (2 * c.R * c.V) + c.h_ev / c.V;
            st->efield = 0;
        }
    }
    if (fmin > st->gfmin * 1.005) st->hsearch = 0;
    if (i < cap) hist[i] = make_double2(xmin, fmin);
    st->last_x = xmin;
    st->last_f = fmin;
    st->interval = interval;
    st->count = i + 1;
}

__global__ void __launch_bounds__(LO_THREADS) k_profile_min(const double* __restrict__ h, LiftoffCfg c,
                                                            double* out) {
    extern __shared__ double lsm[];
    profile_min_block(h, c, lsm, out);
}

__global__ void k_liftoff_reset(LiftoffState* st) {
    LiftoffState z{};
    z.gfmin = DBL_MAX;
    z.gimin = -1;
    z.hsearch = 1;
    z.efield = 1;
    *st = z;
}

size_t smem_bytes(int m) { return sizeof(double) * (3 * size_t(m) + 1); }

}  // namespace

int liftoff_config(int m, double ax, double dx, int mode, int every, double R, double V, LiftoffCfg* c) {
    if (m < 2 || m > LIFTOFF_MAX_M || every < 1 ||
        (mode != VDI_LIFTOFF_SMOOTHED && mode != VDI_LIFTOFF_RAW)) {
        set_error("lift-off analysis: bad options (m %d, mode %d, every %d)", m, mode, every);
        return VDI_ERR_INVALID_ARGUMENT;
    }
    *c = LiftoffCfg{};
    c->m = m;
    c->mode = mode;
    c->every = every;
    c->ax = ax;
    c->dx = dx;
    c->R = R;
    c->V = V;
    c->h_ev = double(500e-9f);                       // tt_analysis.cc:16
    // Gaussian weights of smooth() (tt_analysis.cc:37-47) with its float
    // variables; the spacing is that of the float32 positions.
    const float x0 = float(ax + 0.5 * dx), x1 = float(ax + (m - 0.5) * dx);
    const double adx = (double(x1) - double(x0)) / (m - 1);
    const float glen = 1.2e-6f, gaussian_fac = 7.f;
    float sls = float(glen / adx), fac = float(0.5 / (sls * sls)), v = 0.5f;
    const int cut = int(sls * gaussian_fac) + 1;
    if (mode == VDI_LIFTOFF_SMOOTHED && cut > LIFTOFF_MAX_CUT) {
        set_error("lift-off analysis: smoothing half-width %d exceeds %d (grid too fine)", cut, LIFTOFF_MAX_CUT);
        return VDI_ERR_UNSUPPORTED_SIZE;
    }
    c->cut = cut;
    std::vector<double> w(cut + 1);
    for (int i = 1; i <= cut; i++) {
        w[i] = std::exp(double(-fac * i * i));
        v = float(double(v) + w[i]);
    }
    v = float(0.5 / v);
    w[0] = v;
    for (int i = 1; i <= cut; i++) w[i] *= v;
    for (int i = 0; i <= cut; i++) c->w[cut + i] = c->w[cut - i] = w[i];
    return VDI_OK;
}

int liftoff_reset_async(cudaStream_t s, LiftoffState* st) {
    k_liftoff_reset<<<1, 1, 0, s>>>(st);
    VDI_CUDA(cudaGetLastError());
    return VDI_OK;
}

int liftoff_launch(cudaStream_t s, const double* h, const LiftoffCfg& c, LiftoffState* st, double2* hist, long cap,
                   double dt) {
    static bool attr = false;
    if (!attr) {
        VDI_CUDA(cudaFuncSetAttribute(k_liftoff, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(smem_bytes(LIFTOFF_MAX_M))));
        attr = true;
    }
    k_liftoff<<<1, LO_THREADS, smem_bytes(c.m), s>>>(h, c, st, hist, cap, dt);
    VDI_CUDA(cudaGetLastError());
    return VDI_OK;
}

}  // namespace vdi

using namespace vdi;

extern "C" int vdi_profile_min(int m, double ax, double dx, int mode, const double* d_h, void* stream,
                               double* h_xmin, double* h_fmin) {
    if (!d_h || !h_xmin || !h_fmin) return VDI_ERR_INVALID_ARGUMENT;
    LiftoffCfg c;
    VDI_TRY(liftoff_config(m, ax, dx, mode, 1, 1., 1., &c));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    static bool attr = false;
    if (!attr) {
        VDI_CUDA(cudaFuncSetAttribute(k_profile_min, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(smem_bytes(LIFTOFF_MAX_M))));
        attr = true;
    }
    double* d_out = nullptr;
    VDI_CUDA(cudaMallocAsync(&d_out, 2 * sizeof(double), s));
    k_profile_min<<<1, LO_THREADS, smem_bytes(m), s>>>(d_h, c, d_out);
    cudaError_t e = cudaGetLastError();
    double r[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(r, d_out, sizeof(r), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d_out, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    VDI_CUDA(e);
    *h_xmin = r[0];
    *h_fmin = r[1];
    return VDI_OK;
}
