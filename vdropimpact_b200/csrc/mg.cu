// Geometric multigrid for the four linear systems of the step:
//   MAC projection   (mgs_mac.hh:25-50)      cell-centred 5-point
//   viscous u and v  (visco_impl.hh:28-53)   cell-centred 5-point
//   FEM projection   (mgs_fem.hh:42-57,
//                     mgs_fem.cc:32-53)      node-centred 9-point
//
// Cell-centred systems coarsen 2x2 cells into one, rediscretise the operator
// (coupling coefficients divided by 4 per level, same boundary rows), restrict
// by averaging and prolong bilinearly with ghost values that follow each
// side's boundary condition. Smoothing is red-black Gauss-Seidel.
// The FEM system coarsens node 2I to node I; with bilinear prolongation P and
// restriction P^T the Galerkin operator P^T A P of the bilinear element
// stencil is the same stencil, so every level reuses the fine coefficients.
// Smoothing is four-colour Gauss-Seidel, a true Gauss-Seidel ordering for a
// 9-point stencil. The bottom (liquid-gas) row is a Dirichlet row on every
// level.
//
// Levels with many points run as one launch per operation over the whole
// grid; once the remaining levels fit in shared memory, a single CTA runs the
// rest of the V-cycle there. Solves end when ||b-Az||_2 <= rtol*||b||_2.
// FP32 V-cycles inside FP64 iterative refinement reuse the same kernels with
// T = float.
#include "vdi_internal.hh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace vdi {

static constexpr int MAXLEV = 16;
static constexpr int CTA_THREADS = 1024;
static constexpr size_t CTA_SMEM_LIMIT = 200 * 1024;

// ------------------------------------------------------------------ reduce
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

/** Sum over the block; the result is valid in thread 0. */
__device__ double block_sum(double v) {
    __shared__ double ws[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) ws[w] = v;
    __syncthreads();
    double r = 0;
    if (w == 0) {
        r = lane < int(blockDim.x >> 5) ? ws[lane] : 0.;
        r = warp_sum(r);
    }
    return r;
}

/** Called by every thread of every block with the block's sum in thread 0.
 * Returns true in the last block to finish, whose thread 0 then holds the
 * total summed over the partials in index order (deterministic). */
__device__ bool grid_sum(double blocksum, Reduce rd, double* total) {
    __shared__ int last;
    if (threadIdx.x == 0) {
        rd.partials[blockIdx.x] = blocksum;
        __threadfence();
        unsigned t = atomicAdd(rd.counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double s = 0;
    for (int k = threadIdx.x; k < int(gridDim.x); k += blockDim.x)
        s += __ldcg(rd.partials + k);
    s = block_sum(s);
    if (threadIdx.x == 0) {
        *total = s;
        *rd.counter = 0;
    }
    return true;
}

int reduce_alloc(Reduce& r, int max_blocks) {
    r.max_blocks = max_blocks;
    VDI_CUDA(cudaMalloc(&r.partials, sizeof(double) * max_blocks));
    VDI_CUDA(cudaMalloc(&r.counter, sizeof(unsigned)));
    VDI_CUDA(cudaMemset(r.counter, 0, sizeof(unsigned)));
    return VDI_OK;
}

void reduce_free(Reduce& r) {
    if (r.partials) cudaFree(r.partials);
    if (r.counter) cudaFree(r.counter);
    r.partials = nullptr;
    r.counter = nullptr;
}

/** Convergence decision, made by one thread after a residual norm. Sets the
 * graph loop condition when a handle is given. */
__device__ void solve_decide(SolveCtl* ctl, double r2, int count_cycle, int use_cond,
                             cudaGraphConditionalHandle h) {
    if (count_cycle) ctl->it += 1;
    ctl->rnorm2 = r2;
    int cont = 0;
    double thr = ctl->rtol * ctl->rtol * ctl->bnorm2;
    if (!(r2 <= thr)) {
        if (!isfinite(r2)) {
            ctl->status |= DEV_NONFINITE;
        } else if (ctl->it >= ctl->max_it) {
            ctl->status |= DEV_MG_NOT_CONVERGED;
        } else {
            cont = 1;
        }
    }
    if (ctl->status) ctl->sticky |= ctl->status;
    if (!cont) {
        ctl->done = 1;
        ctl->solves += 1;
        ctl->vcycles += ctl->it;
        ctl->last_rel = ctl->bnorm2 > 0 ? sqrt(r2 / ctl->bnorm2) : 0.;
    }
    if (use_cond) cudaGraphSetConditional(h, cont);
}

// ------------------------------------------------------- cell-centred ops
template <typename T>
struct CCc {
    int m, n;
    T ox, oy;          // off-diagonal couplings of A
    T d[3][3];         // diagonal by (x class, y class): 0 first, 1 interior, 2 last
    T invd[3][3];
    signed char gL, gR, gD, gU;
};

__device__ __forceinline__ int cls(int i, int m) { return i == 0 ? 0 : (i == m - 1 ? 2 : 1); }

/** A z at (i,j) for a grid array with pitch m (neighbours outside the grid
 * do not contribute, as in mul_a of mgs_mac.hh:39-45 / visco_impl.hh:40-46). */
template <typename T>
__device__ __forceinline__ T cc_off(const CCc<T>& c, const T* z, int i, int j) {
    int ij = i + c.m * j;
    T xs = (i > 0 ? z[ij - 1] : T(0)) + (i < c.m - 1 ? z[ij + 1] : T(0));
    T ys = (j > 0 ? z[ij - c.m] : T(0)) + (j < c.n - 1 ? z[ij + c.m] : T(0));
    return c.ox * xs + c.oy * ys;
}

template <typename T>
__device__ __forceinline__ T cc_resid(const CCc<T>& c, const T* z, const T* b, int i, int j) {
    int ij = i + c.m * j;
    return b[ij] - c.d[cls(i, c.m)][cls(j, c.n)] * z[ij] - cc_off(c, z, i, j);
}

template <typename T>
__device__ __forceinline__ void cc_relax(const CCc<T>& c, T* z, const T* b, int i, int j) {
    int ij = i + c.m * j;
    z[ij] = (b[ij] - cc_off(c, z, i, j)) * c.invd[cls(i, c.m)][cls(j, c.n)];
}

/** Bilinear cell-centred prolongation of the coarse correction to fine cell
 * (i,j); ghost values are g * (boundary value) on each side. */
template <typename T>
__device__ __forceinline__ T cc_interp(const CCc<T>& f, const T* zc, int mc, int nc, int i, int j) {
    int I = i >> 1, J = j >> 1;
    int sx = (i & 1) ? 1 : -1, sy = (j & 1) ? 1 : -1;
    int Ix = I + sx, Jy = J + sy;
    bool xo = Ix < 0 || Ix >= mc, yo = Jy < 0 || Jy >= nc;
    T gx = T(sx < 0 ? f.gL : f.gR), gy = T(sy < 0 ? f.gD : f.gU);
    T c00 = zc[I + mc * J];
    T c10 = xo ? gx * c00 : zc[Ix + mc * J];
    T c01 = yo ? gy * c00 : zc[I + mc * Jy];
    T c11;
    if (xo && yo) c11 = gx * gy * c00;
    else if (xo) c11 = gx * c01;
    else if (yo) c11 = gy * c10;
    else c11 = zc[Ix + mc * Jy];
    return T(0.5625) * c00 + T(0.1875) * (c10 + c01) + T(0.0625) * c11;
}

template <typename T>
__global__ void cc_rb_sweep(CCc<T> c, T* __restrict__ z, const T* __restrict__ b, int color) {
    int half = c.m >> 1;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= half * c.n) return;
    int j = k / half;
    int i = 2 * (k - j * half) + ((j + color) & 1);
    cc_relax(c, z, b, i, j);
}

template <typename T>
__global__ void cc_resid_restrict(CCc<T> c, const T* __restrict__ z, const T* __restrict__ b,
                                  T* __restrict__ bc) {
    int mc = c.m >> 1, nc = c.n >> 1;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= mc * nc) return;
    int J = k / mc, I = k - J * mc;
    int i = 2 * I, j = 2 * J;
    T s = cc_resid(c, z, b, i, j) + cc_resid(c, z, b, i + 1, j) + cc_resid(c, z, b, i, j + 1) +
          cc_resid(c, z, b, i + 1, j + 1);
    bc[k] = T(0.25) * s;
}

template <typename T>
__global__ void cc_prolong_add(CCc<T> f, T* __restrict__ z, const T* __restrict__ zc) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= f.m * f.n) return;
    int j = k / f.m, i = k - j * f.m;
    z[k] += cc_interp(f, zc, f.m >> 1, f.n >> 1, i, j);
}

/** ||b - A z||^2 (accumulated in FP64) followed by the solve decision. */
template <typename T>
__global__ void cc_resid_norm(CCc<T> c, const T* __restrict__ z, const T* __restrict__ b, Reduce rd,
                              SolveCtl* ctl, int count_cycle, int use_cond,
                              cudaGraphConditionalHandle h) {
    double s = 0;
    int tot = c.m * c.n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += gridDim.x * blockDim.x) {
        int j = k / c.m, i = k - j * c.m;
        double r = double(cc_resid(c, z, b, i, j));
        s += r * r;
    }
    s = block_sum(s);
    double total;
    if (grid_sum(s, rd, &total) && threadIdx.x == 0) solve_decide(ctl, total, count_cycle, use_cond, h);
}

/** FP64 residual of an FP64 iterate written as FP32 (the refinement step),
 * with its FP64 norm and the solve decision. */
__global__ void cc_resid_to32(CCc<double> c, const double* __restrict__ z, const double* __restrict__ b,
                              float* __restrict__ r32, Reduce rd, SolveCtl* ctl, int count_cycle,
                              int use_cond, cudaGraphConditionalHandle h) {
    double s = 0;
    int tot = c.m * c.n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += gridDim.x * blockDim.x) {
        int j = k / c.m, i = k - j * c.m;
        double r = cc_resid(c, z, b, i, j);
        r32[k] = float(r);
        s += r * r;
    }
    s = block_sum(s);
    double total;
    if (grid_sum(s, rd, &total) && threadIdx.x == 0) solve_decide(ctl, total, count_cycle, use_cond, h);
}

template <typename T>
__global__ void cc_apply(CCc<T> c, const T* __restrict__ z, T* __restrict__ y) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.m * c.n) return;
    int j = k / c.m, i = k - j * c.m;
    y[k] = c.d[cls(i, c.m)][cls(j, c.n)] * z[k] + cc_off(c, z, i, j);
}

template <typename T>
__global__ void cc_residual_out(CCc<T> c, const T* __restrict__ z, const T* __restrict__ b, T* __restrict__ r) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.m * c.n) return;
    int j = k / c.m, i = k - j * c.m;
    r[k] = cc_resid(c, z, b, i, j);
}

/** The remaining levels of a cell-centred V-cycle inside one CTA: level 0
 * of the descriptor reads b (and z unless zero_init) from global memory and
 * writes z back; every array lives in shared memory. */
template <typename T>
struct CCStack {
    int nl;
    CCc<T> lv[MAXLEV];
    int off[MAXLEV];     // element offsets of z_l; b_l follows z_l
    int nu1, nu2, ncoarse;
};

template <typename T>
__device__ void cta_cc_sweep(const CCc<T>& c, T* z, const T* b, int color) {
    int tot = c.m * c.n;
    for (int k = threadIdx.x; k < tot; k += blockDim.x) {
        int j = k / c.m, i = k - j * c.m;
        if (((i + j) & 1) == color) cc_relax(c, z, b, i, j);
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(CTA_THREADS) cc_cta_cycle(CCStack<T> st, const T* __restrict__ gb,
                                                           T* __restrict__ gz, int zero_init) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    {
        const CCc<T>& c0 = st.lv[0];
        T* z = sm + st.off[0];
        T* b = z + c0.m * c0.n;
        int tot = c0.m * c0.n;
        for (int k = threadIdx.x; k < tot; k += blockDim.x) {
            b[k] = gb[k];
            z[k] = zero_init ? T(0) : gz[k];
        }
    }
    __syncthreads();
    // descend
    for (int l = 0; l < st.nl - 1; l++) {
        const CCc<T>& c = st.lv[l];
        T* z = sm + st.off[l];
        T* b = z + c.m * c.n;
        if (l > 0) {
            for (int k = threadIdx.x; k < c.m * c.n; k += blockDim.x) z[k] = T(0);
            __syncthreads();
        }
        for (int s = 0; s < st.nu1; s++) {
            cta_cc_sweep(c, z, b, 0);
            cta_cc_sweep(c, z, b, 1);
        }
        const CCc<T>& cc = st.lv[l + 1];
        T* bcn = sm + st.off[l + 1] + cc.m * cc.n;
        for (int k = threadIdx.x; k < cc.m * cc.n; k += blockDim.x) {
            int J = k / cc.m, I = k - J * cc.m;
            int i = 2 * I, j = 2 * J;
            T s = cc_resid(c, z, b, i, j) + cc_resid(c, z, b, i + 1, j) + cc_resid(c, z, b, i, j + 1) +
                  cc_resid(c, z, b, i + 1, j + 1);
            bcn[k] = T(0.25) * s;
        }
        __syncthreads();
    }
    // coarsest: plain sweeps from zero
    {
        int l = st.nl - 1;
        const CCc<T>& c = st.lv[l];
        T* z = sm + st.off[l];
        T* b = z + c.m * c.n;
        if (l > 0) {
            for (int k = threadIdx.x; k < c.m * c.n; k += blockDim.x) z[k] = T(0);
            __syncthreads();
        }
        int ns = (l > 0) ? st.ncoarse : st.nu1 + st.nu2;
        for (int s = 0; s < ns; s++) {
            cta_cc_sweep(c, z, b, 0);
            cta_cc_sweep(c, z, b, 1);
        }
    }
    // ascend
    for (int l = st.nl - 2; l >= 0; l--) {
        const CCc<T>& c = st.lv[l];
        T* z = sm + st.off[l];
        T* b = z + c.m * c.n;
        const T* zc = sm + st.off[l + 1];
        for (int k = threadIdx.x; k < c.m * c.n; k += blockDim.x) {
            int j = k / c.m, i = k - j * c.m;
            z[k] += cc_interp(c, zc, c.m >> 1, c.n >> 1, i, j);
        }
        __syncthreads();
        for (int s = 0; s < st.nu2; s++) {
            cta_cc_sweep(c, z, b, 1);
            cta_cc_sweep(c, z, b, 0);
        }
    }
    {
        const CCc<T>& c0 = st.lv[0];
        const T* z = sm + st.off[0];
        for (int k = threadIdx.x; k < c0.m * c0.n; k += blockDim.x) gz[k] = z[k];
    }
}

// ------------------------------------------------------------- FEM ops
template <typename T>
struct FEMc {
    int M, N;
    T fm, fey, hey, fex, hex, fc;
    T d[3][3], invd[3][3];
};

/** mul_a of mgs_fem.cc:32-53 on a grid array with pitch M. */
template <typename T>
__device__ __forceinline__ T fem_off(const FEMc<T>& c, const T* z, int i, int j) {
    if (j == 0) return T(0);
    const int M = c.M;
    const T* w = z + i + M * j;
    const T* wm = w - M;
    if (j == c.N - 1) {
        if (i == 0) return c.fc * wm[1] + c.hey * (*wm) + c.hex * w[1];
        if (i == M - 1) return c.fc * wm[-1] + c.hey * (*wm) + c.hex * w[-1];
        return c.fc * (wm[-1] + wm[1]) + c.fey * (*wm) + c.hex * (w[-1] + w[1]);
    }
    if (i == 0) return c.fc * (wm[1] + w[M + 1]) + c.hey * (*wm + w[M]) + c.fex * w[1];
    if (i == M - 1) return c.fc * (wm[-1] + w[M - 1]) + c.hey * (*wm + w[M]) + c.fex * w[-1];
    return c.fc * (wm[-1] + wm[1] + w[M - 1] + w[M + 1]) + c.fey * (*wm + w[M]) + c.fex * (w[-1] + w[1]);
}

template <typename T>
__device__ __forceinline__ T fem_resid(const FEMc<T>& c, const T* z, const T* b, int i, int j) {
    int ij = i + c.M * j;
    return b[ij] - c.d[cls(i, c.M)][cls(j, c.N)] * z[ij] - fem_off(c, z, i, j);
}

template <typename T>
__device__ __forceinline__ void fem_relax(const FEMc<T>& c, T* z, const T* b, int i, int j) {
    int ij = i + c.M * j;
    z[ij] = (b[ij] - fem_off(c, z, i, j)) * c.invd[cls(i, c.M)][cls(j, c.N)];
}

/** P^T r at coarse node (I,J); zero on the Dirichlet bottom row. */
template <typename T>
__device__ __forceinline__ T fem_restrict_at(int M, int N, const T* r, int I, int J) {
    if (J == 0) return T(0);
    T s = 0;
    for (int dj = -1; dj <= 1; dj++) {
        int j = 2 * J + dj;
        if (j < 0 || j >= N) continue;
        T wy = dj == 0 ? T(1) : T(0.5);
        for (int di = -1; di <= 1; di++) {
            int i = 2 * I + di;
            if (i < 0 || i >= M) continue;
            T wx = di == 0 ? T(1) : T(0.5);
            s += wx * wy * r[i + M * j];
        }
    }
    return s;
}

/** Bilinear prolongation of node-centred corrections to fine node (i,j). */
template <typename T>
__device__ __forceinline__ T fem_interp(const T* zc, int Mc, int i, int j) {
    int I = i >> 1, J = j >> 1;
    bool ox = i & 1, oy = j & 1;
    T c00 = zc[I + Mc * J];
    if (!ox && !oy) return c00;
    if (ox && !oy) return T(0.5) * (c00 + zc[I + 1 + Mc * J]);
    if (!ox && oy) return T(0.5) * (c00 + zc[I + Mc * (J + 1)]);
    return T(0.25) * (c00 + zc[I + 1 + Mc * J] + zc[I + Mc * (J + 1)] + zc[I + 1 + Mc * (J + 1)]);
}

template <typename T>
__global__ void fem_color_sweep(FEMc<T> c, T* __restrict__ z, const T* __restrict__ b, int ci, int cj) {
    int mx = (c.M - ci + 1) >> 1, my = (c.N - cj + 1) >> 1;
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= mx * my) return;
    int q = k / mx;
    int i = ci + 2 * (k - q * mx), j = cj + 2 * q;
    fem_relax(c, z, b, i, j);
}

template <typename T>
__global__ void fem_residual_k(FEMc<T> c, const T* __restrict__ z, const T* __restrict__ b, T* __restrict__ r) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.M * c.N) return;
    int j = k / c.M, i = k - j * c.M;
    r[k] = fem_resid(c, z, b, i, j);
}

template <typename T>
__global__ void fem_restrict_k(int M, int N, const T* __restrict__ r, int Mc, int Nc, T* __restrict__ bc) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Mc * Nc) return;
    int J = k / Mc, I = k - J * Mc;
    bc[k] = fem_restrict_at(M, N, r, I, J);
}

template <typename T>
__global__ void fem_prolong_add(int M, int N, T* __restrict__ z, int Mc, const T* __restrict__ zc) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M * N) return;
    int j = k / M, i = k - j * M;
    if (j == 0) return;
    z[k] += fem_interp(zc, Mc, i, j);
}

template <typename T>
__global__ void fem_resid_norm(FEMc<T> c, const T* __restrict__ z, const T* __restrict__ b, Reduce rd,
                               SolveCtl* ctl, int count_cycle, int use_cond, cudaGraphConditionalHandle h) {
    double s = 0;
    int tot = c.M * c.N;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += gridDim.x * blockDim.x) {
        int j = k / c.M, i = k - j * c.M;
        double r = double(fem_resid(c, z, b, i, j));
        s += r * r;
    }
    s = block_sum(s);
    double total;
    if (grid_sum(s, rd, &total) && threadIdx.x == 0) solve_decide(ctl, total, count_cycle, use_cond, h);
}

__global__ void fem_resid_to32(FEMc<double> c, const double* __restrict__ z, const double* __restrict__ b,
                               float* __restrict__ r32, Reduce rd, SolveCtl* ctl, int count_cycle,
                               int use_cond, cudaGraphConditionalHandle h) {
    double s = 0;
    int tot = c.M * c.N;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += gridDim.x * blockDim.x) {
        int j = k / c.M, i = k - j * c.M;
        double r = fem_resid(c, z, b, i, j);
        r32[k] = float(r);
        s += r * r;
    }
    s = block_sum(s);
    double total;
    if (grid_sum(s, rd, &total) && threadIdx.x == 0) solve_decide(ctl, total, count_cycle, use_cond, h);
}

template <typename T>
__global__ void fem_apply(FEMc<T> c, const T* __restrict__ z, T* __restrict__ y) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c.M * c.N) return;
    int j = k / c.M, i = k - j * c.M;
    y[k] = c.d[cls(i, c.M)][cls(j, c.N)] * z[k] + fem_off(c, z, i, j);
}

template <typename T>
struct FEMStack {
    int nl;
    FEMc<T> lv[MAXLEV];
    int off[MAXLEV];     // z_l, then b_l, then r_l
    int nu1, nu2, ncoarse;
};

template <typename T>
__device__ void cta_fem_sweep(const FEMc<T>& c, T* z, const T* b, int color) {
    int ci = color & 1, cj = color >> 1;
    int tot = c.M * c.N;
    for (int k = threadIdx.x; k < tot; k += blockDim.x) {
        int j = k / c.M, i = k - j * c.M;
        if ((i & 1) == ci && (j & 1) == cj) fem_relax(c, z, b, i, j);
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(CTA_THREADS) fem_cta_cycle(FEMStack<T> st, const T* __restrict__ gb,
                                                            T* __restrict__ gz, int zero_init) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    {
        const FEMc<T>& c0 = st.lv[0];
        T* z = sm + st.off[0];
        T* b = z + c0.M * c0.N;
        for (int k = threadIdx.x; k < c0.M * c0.N; k += blockDim.x) {
            b[k] = gb[k];
            z[k] = zero_init ? T(0) : gz[k];
        }
    }
    __syncthreads();
    for (int l = 0; l < st.nl - 1; l++) {
        const FEMc<T>& c = st.lv[l];
        int tot = c.M * c.N;
        T* z = sm + st.off[l];
        T* b = z + tot;
        T* r = b + tot;
        if (l > 0) {
            for (int k = threadIdx.x; k < tot; k += blockDim.x) z[k] = T(0);
            __syncthreads();
        }
        for (int s = 0; s < st.nu1; s++)
            for (int q = 0; q < 4; q++) cta_fem_sweep(c, z, b, q);
        for (int k = threadIdx.x; k < tot; k += blockDim.x) {
            int j = k / c.M, i = k - j * c.M;
            r[k] = fem_resid(c, z, b, i, j);
        }
        __syncthreads();
        const FEMc<T>& cc = st.lv[l + 1];
        T* bcn = sm + st.off[l + 1] + cc.M * cc.N;
        for (int k = threadIdx.x; k < cc.M * cc.N; k += blockDim.x) {
            int J = k / cc.M, I = k - J * cc.M;
            bcn[k] = fem_restrict_at(c.M, c.N, r, I, J);
        }
        __syncthreads();
    }
    {
        int l = st.nl - 1;
        const FEMc<T>& c = st.lv[l];
        T* z = sm + st.off[l];
        T* b = z + c.M * c.N;
        if (l > 0) {
            for (int k = threadIdx.x; k < c.M * c.N; k += blockDim.x) z[k] = T(0);
            __syncthreads();
        }
        int ns = (l > 0) ? st.ncoarse : st.nu1 + st.nu2;
        for (int s = 0; s < ns; s++)
            for (int q = 0; q < 4; q++) cta_fem_sweep(c, z, b, q);
    }
    for (int l = st.nl - 2; l >= 0; l--) {
        const FEMc<T>& c = st.lv[l];
        int tot = c.M * c.N;
        T* z = sm + st.off[l];
        T* b = z + tot;
        const T* zc = sm + st.off[l + 1];
        for (int k = threadIdx.x; k < tot; k += blockDim.x) {
            int j = k / c.M, i = k - j * c.M;
            if (j > 0) z[k] += fem_interp(zc, st.lv[l + 1].M, i, j);
        }
        __syncthreads();
        for (int s = 0; s < st.nu2; s++)
            for (int q = 3; q >= 0; q--) cta_fem_sweep(c, z, b, q);
    }
    {
        const FEMc<T>& c0 = st.lv[0];
        const T* z = sm + st.off[0];
        for (int k = threadIdx.x; k < c0.M * c0.N; k += blockDim.x) gz[k] = z[k];
    }
}

// ------------------------------------------------------------ misc kernels
__global__ void norm2_kernel(const double* __restrict__ x, int n, Reduce rd, SolveCtl* ctl) {
    double s = 0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) s += x[k] * x[k];
    s = block_sum(s);
    double total;
    if (grid_sum(s, rd, &total) && threadIdx.x == 0) {
        ctl->bnorm2 = total;
        ctl->it = 0;
        ctl->done = 0;
        ctl->status = 0;
    }
}

/** If ||b|| = 0 the solution is z = 0 (the shim and this library agree on
 * that convention); zero z once the norm is known. */
__global__ void zero_if_b_zero(double* __restrict__ z, int n, const SolveCtl* ctl) {
    if (ctl->bnorm2 != 0.) return;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) z[k] = 0.;
}

__global__ void add_f32_to_f64(double* __restrict__ z, const float* __restrict__ e, int n) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) z[k] += double(e[k]);
}

__global__ void norm_result(const Reduce rd, double* out) {}

/** Writes the final residual norm of a standalone residual computation. */
template <typename T>
__global__ void resid_norm_plain(int kind, CCc<T> cc, FEMc<T> fc, const T* z, const T* b, T* r, Reduce rd,
                                 double* out) {
    double s = 0;
    int tot = kind == VDI_MG_FEM ? fc.M * fc.N : cc.m * cc.n;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += gridDim.x * blockDim.x) {
        double v;
        if (kind == VDI_MG_FEM) {
            int j = k / fc.M, i = k - j * fc.M;
            v = double(fem_resid(fc, z, b, i, j));
        } else {
            int j = k / cc.m, i = k - j * cc.m;
            v = double(cc_resid(cc, z, b, i, j));
        }
        if (r) r[k] = T(v);
        s += v * v;
    }
    s = block_sum(s);
    double total;
    if (grid_sum(s, rd, &total) && threadIdx.x == 0) *out = sqrt(total);
}

// =================================================================== host
static inline int nblk(long n, int t = 256) { return int((n + t - 1) / t); }

/** Per-level description in double precision, converted per precision. */
struct LevelD {
    int m, n;              // cell-centred: cells; FEM: nodes (M, N)
    double ox, oy;         // cell-centred couplings
    double d[3][3];
    signed char gL, gR, gD, gU;
};

class MG {
  public:
    int kind = 0;
    int m = 0, n = 0;      // fine grid of the problem class (cells or nodes)
    double c1 = 0, c2 = 0; // dx,dy (MAC/FEM) or vfx,vfy (viscous)
    int x_sym = 0;
    std::vector<LevelD> lv;
    FEMOp fop{};
    int nlev = 0;
    int nmulti64 = 0, nmulti32 = 0;
    size_t smem64 = 0, smem32 = 0;
    // device buffers: index l holds level l (level 0 of z64/b64 is the caller's)
    std::vector<double*> z64, b64, r64;
    std::vector<float*> z32, b32, r32;
    Reduce rd;
    SolveCtl* ctl = nullptr;
    int nu1 = 2, nu2 = 2;
    double rtol = 1e-10;
    int max_it = 200;

    ~MG() { release(); }

    void release() {
        for (auto p : z64) if (p) cudaFree(p);
        for (auto p : b64) if (p) cudaFree(p);
        for (auto p : r64) if (p) cudaFree(p);
        for (auto p : z32) if (p) cudaFree(p);
        for (auto p : b32) if (p) cudaFree(p);
        for (auto p : r32) if (p) cudaFree(p);
        z64.clear(); b64.clear(); r64.clear(); z32.clear(); b32.clear(); r32.clear();
        reduce_free(rd);
        if (ctl) cudaFree(ctl);
        ctl = nullptr;
    }

    long size(int l) const { return long(lv[l].m) * lv[l].n; }

    /** Diagonals and couplings of level l, matching the problem classes'
     * a_cc / mul_a (mgs_mac.hh:33-45, visco_impl.hh:36-46) with the level's
     * scaled coefficients. */
    void fill_cc(LevelD& L, double kx, double ky) {
        L.ox = kind == VDI_MG_MAC ? kx : -kx;
        L.oy = kind == VDI_MG_MAC ? ky : -ky;
        bool horiz = kind == VDI_MG_VISC_U;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                double v;
                if (kind == VDI_MG_MAC) {
                    double xp = a == 1 ? -2 * kx : -kx;
                    if (L.m == 1) xp = -kx;
                    double yp = b == 0 ? -3 * ky : (b == 1 ? -2 * ky : -ky);
                    v = xp + yp;
                } else {
                    double yp = b == 0 ? vfy_part(ky, true) : 2 * ky;
                    if (x_sym) {
                        double xp = a == 0 ? (horiz ? 3 * kx : kx) : 2 * kx;
                        v = 1 + xp + yp;
                    } else {
                        v = 1 + 2 * kx + yp;
                    }
                }
                L.d[a][b] = v;
            }
        if (kind == VDI_MG_MAC) {
            L.gL = 1; L.gR = 1; L.gD = -1; L.gU = 1;
        } else {
            L.gL = x_sym ? (horiz ? -1 : 1) : 0;
            L.gR = 0; L.gD = 1; L.gU = 0;
        }
    }
    static double vfy_part(double ky, bool bottom) { return bottom ? ky : 2 * ky; }

    void fill_fem(LevelD& L) {
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                L.d[a][b] = (a == 1 ? 1. : 0.5) * (b == 1 ? 1. : 0.5) * fop.fm;
    }

    template <typename T>
    CCc<T> ccc(int l) const {
        const LevelD& L = lv[l];
        CCc<T> c;
        c.m = L.m; c.n = L.n;
        c.ox = T(L.ox); c.oy = T(L.oy);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                c.d[a][b] = T(L.d[a][b]);
                c.invd[a][b] = T(1.0 / L.d[a][b]);
            }
        c.gL = L.gL; c.gR = L.gR; c.gD = L.gD; c.gU = L.gU;
        return c;
    }

    template <typename T>
    FEMc<T> femc(int l) const {
        const LevelD& L = lv[l];
        FEMc<T> c;
        c.M = L.m; c.N = L.n;
        c.fm = T(fop.fm); c.fey = T(fop.fey); c.hey = T(fop.hey);
        c.fex = T(fop.fex); c.hex = T(fop.hex); c.fc = T(fop.fc);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                c.d[a][b] = T(L.d[a][b]);
                c.invd[a][b] = T(1.0 / L.d[a][b]);
            }
        return c;
    }

    int build_levels() {
        lv.clear();
        if (kind == VDI_MG_FEM) {
            double dydx = c2 / c1, dxdy = c1 / c2;
            // mgs_fem.cc:8-11
            fop.fm = 4. / 3. * (dxdy + dydx);
            fop.fey = 1. / 3. * (-2 * dxdy + dydx);
            fop.hey = 0.5 * fop.fey;
            fop.fex = 1. / 3. * (-2 * dydx + dxdy);
            fop.hex = 0.5 * fop.fex;
            fop.fc = -1. / 6. * (dxdy + dydx);
            int M = m, N = n;
            while (true) {
                LevelD L{};
                L.m = M; L.n = N;
                fill_fem(L);
                lv.push_back(L);
                if (M < 5 || N < 5 || ((M - 1) & 1) || ((N - 1) & 1) || int(lv.size()) == MAXLEV) break;
                M = (M - 1) / 2 + 1;
                N = (N - 1) / 2 + 1;
            }
        } else {
            double kx, ky;
            kx = c1;   // MAC: xxsp, yysp; viscous: vfx, vfy
            ky = c2;
            int mm = m, nn = n;
            while (true) {
                LevelD L{};
                L.m = mm; L.n = nn;
                fill_cc(L, kx, ky);
                lv.push_back(L);
                if ((mm & 1) || (nn & 1) || mm < 4 || nn < 2 || int(lv.size()) == MAXLEV) break;
                mm >>= 1; nn >>= 1;
                kx *= 0.25; ky *= 0.25;
            }
        }
        nlev = int(lv.size());
        // the CTA-resident tail must fit in shared memory
        int arrays = kind == VDI_MG_FEM ? 3 : 2;
        auto tail_bytes = [&](int from, size_t es) {
            size_t t = 0;
            for (int l = from; l < nlev; l++) t += size_t(arrays) * size(l) * es;
            return t;
        };
        nmulti64 = -1;
        for (int l = 0; l < nlev; l++)
            if (tail_bytes(l, 8) <= CTA_SMEM_LIMIT) { nmulti64 = l; break; }
        nmulti32 = -1;
        for (int l = 0; l < nlev; l++)
            if (tail_bytes(l, 4) <= CTA_SMEM_LIMIT) { nmulti32 = l; break; }
        if (nmulti64 < 0 || nmulti32 < 0) {
            set_error("multigrid: %dx%d grid does not coarsen to a shared-memory-sized level", m, n);
            return VDI_ERR_UNSUPPORTED_SIZE;
        }
        smem64 = tail_bytes(nmulti64, 8);
        smem32 = tail_bytes(nmulti32, 4);
        return VDI_OK;
    }

    int alloc() {
        z64.assign(nlev, nullptr); b64.assign(nlev, nullptr); r64.assign(nlev, nullptr);
        z32.assign(nlev, nullptr); b32.assign(nlev, nullptr); r32.assign(nlev, nullptr);
        for (int l = 0; l < nlev; l++) {
            size_t s = size_t(size(l));
            if (l > 0 && l <= nmulti64) {
                VDI_CUDA(cudaMalloc(&z64[l], s * 8));
                VDI_CUDA(cudaMalloc(&b64[l], s * 8));
            }
            if (kind == VDI_MG_FEM && l < nmulti64) VDI_CUDA(cudaMalloc(&r64[l], s * 8));
            if (l <= nmulti32) {
                VDI_CUDA(cudaMalloc(&z32[l], s * 4));
                VDI_CUDA(cudaMalloc(&b32[l], s * 4));
            }
            if (kind == VDI_MG_FEM && l < nmulti32) VDI_CUDA(cudaMalloc(&r32[l], s * 4));
        }
        VDI_TRY(reduce_alloc(rd, 1024));
        VDI_CUDA(cudaMalloc(&ctl, sizeof(SolveCtl)));
        VDI_CUDA(cudaMemset(ctl, 0, sizeof(SolveCtl)));
        VDI_TRY(set_ctl_params(0, rtol, max_it));
        VDI_CUDA(cudaFuncSetAttribute(cc_cta_cycle<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(CTA_SMEM_LIMIT)));
        VDI_CUDA(cudaFuncSetAttribute(cc_cta_cycle<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(CTA_SMEM_LIMIT)));
        VDI_CUDA(cudaFuncSetAttribute(fem_cta_cycle<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(CTA_SMEM_LIMIT)));
        VDI_CUDA(cudaFuncSetAttribute(fem_cta_cycle<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(CTA_SMEM_LIMIT)));
        return VDI_OK;
    }

    int ncoarse_sweeps(int l) const {
        long s = long(lv[l].m) + lv[l].n;
        long v = 4 * s * s;
        return int(std::min(400L, std::max(20L, v)));
    }

    /** One V-cycle on level l (precision T). z/b are level-l arrays. */
    template <typename T>
    int vcycle(cudaStream_t s, int l, const T* b, T* z, int nmulti, std::vector<T*>& zs,
               std::vector<T*>& bs, std::vector<T*>& rs, size_t smem) {
        if (l == nmulti) {
            if (kind == VDI_MG_FEM) {
                FEMStack<T> st{};
                st.nl = nlev - l;
                int off = 0;
                for (int q = 0; q < st.nl; q++) {
                    st.lv[q] = femc<T>(l + q);
                    st.off[q] = off;
                    off += 3 * int(size(l + q));
                }
                st.nu1 = nu1; st.nu2 = nu2; st.ncoarse = ncoarse_sweeps(nlev - 1);
                fem_cta_cycle<T><<<1, CTA_THREADS, smem, s>>>(st, b, z, l > 0);
            } else {
                CCStack<T> st{};
                st.nl = nlev - l;
                int off = 0;
                for (int q = 0; q < st.nl; q++) {
                    st.lv[q] = ccc<T>(l + q);
                    st.off[q] = off;
                    off += 2 * int(size(l + q));
                }
                st.nu1 = nu1; st.nu2 = nu2; st.ncoarse = ncoarse_sweeps(nlev - 1);
                cc_cta_cycle<T><<<1, CTA_THREADS, smem, s>>>(st, b, z, l > 0);
            }
            VDI_CUDA(cudaGetLastError());
            return VDI_OK;
        }
        long N = size(l);
        if (l > 0) VDI_CUDA(cudaMemsetAsync(z, 0, sizeof(T) * N, s));
        if (kind == VDI_MG_FEM) {
            FEMc<T> c = femc<T>(l);
            auto sweep = [&](int q) {
                int ci = q & 1, cj = q >> 1;
                long cnt = long((c.M - ci + 1) >> 1) * ((c.N - cj + 1) >> 1);
                fem_color_sweep<T><<<nblk(cnt), 256, 0, s>>>(c, z, b, ci, cj);
            };
            for (int k = 0; k < nu1; k++)
                for (int q = 0; q < 4; q++) sweep(q);
            fem_residual_k<T><<<nblk(N), 256, 0, s>>>(c, z, b, rs[l]);
            fem_restrict_k<T><<<nblk(size(l + 1)), 256, 0, s>>>(c.M, c.N, rs[l], lv[l + 1].m, lv[l + 1].n,
                                                                 bs[l + 1]);
            VDI_TRY(vcycle<T>(s, l + 1, bs[l + 1], zs[l + 1], nmulti, zs, bs, rs, smem));
            fem_prolong_add<T><<<nblk(N), 256, 0, s>>>(c.M, c.N, z, lv[l + 1].m, zs[l + 1]);
            for (int k = 0; k < nu2; k++)
                for (int q = 3; q >= 0; q--) sweep(q);
        } else {
            CCc<T> c = ccc<T>(l);
            int half = int(N / 2);
            for (int k = 0; k < nu1; k++) {
                cc_rb_sweep<T><<<nblk(half), 256, 0, s>>>(c, z, b, 0);
                cc_rb_sweep<T><<<nblk(half), 256, 0, s>>>(c, z, b, 1);
            }
            cc_resid_restrict<T><<<nblk(size(l + 1)), 256, 0, s>>>(c, z, b, bs[l + 1]);
            VDI_TRY(vcycle<T>(s, l + 1, bs[l + 1], zs[l + 1], nmulti, zs, bs, rs, smem));
            cc_prolong_add<T><<<nblk(N), 256, 0, s>>>(c, z, zs[l + 1]);
            for (int k = 0; k < nu2; k++) {
                cc_rb_sweep<T><<<nblk(half), 256, 0, s>>>(c, z, b, 1);
                cc_rb_sweep<T><<<nblk(half), 256, 0, s>>>(c, z, b, 0);
            }
        }
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    int vcycle64(cudaStream_t s, const double* b, double* z) {
        return vcycle<double>(s, 0, b, z, nmulti64, z64, b64, r64, smem64);
    }
    int vcycle32(cudaStream_t s) {
        return vcycle<float>(s, 0, b32[0], z32[0], nmulti32, z32, b32, r32, smem32);
    }

    int norm_blocks() const { return std::min(rd.max_blocks, std::max(1, nblk(size(0), 256))); }

    /** Enqueue: residual norm of z + decision (FP64 path). */
    int enqueue_resid_norm(cudaStream_t s, const double* b, const double* z, int count_cycle, int use_cond,
                           cudaGraphConditionalHandle h) {
        int nb = std::min(norm_blocks(), 4 * 148);
        if (kind == VDI_MG_FEM)
            fem_resid_norm<double><<<nb, 256, 0, s>>>(femc<double>(0), z, b, rd, ctl, count_cycle, use_cond, h);
        else
            cc_resid_norm<double><<<nb, 256, 0, s>>>(ccc<double>(0), z, b, rd, ctl, count_cycle, use_cond, h);
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    int enqueue_resid32(cudaStream_t s, const double* b, const double* z, int count_cycle, int use_cond,
                        cudaGraphConditionalHandle h) {
        int nb = std::min(norm_blocks(), 4 * 148);
        if (kind == VDI_MG_FEM)
            fem_resid_to32<<<nb, 256, 0, s>>>(femc<double>(0), z, b, b32[0], rd, ctl, count_cycle, use_cond, h);
        else
            cc_resid_to32<<<nb, 256, 0, s>>>(ccc<double>(0), z, b, b32[0], rd, ctl, count_cycle, use_cond, h);
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    int enqueue_begin(cudaStream_t s, const double* b, double* z) {
        int nb = std::min(norm_blocks(), 4 * 148);
        norm2_kernel<<<nb, 256, 0, s>>>(b, int(size(0)), rd, ctl);
        zero_if_b_zero<<<nblk(size(0)), 256, 0, s>>>(z, int(size(0)), ctl);
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    /** One iteration of the solve loop body (precision-dependent). */
    int enqueue_body(cudaStream_t s, const double* b, double* z, int precision, int use_cond,
                     cudaGraphConditionalHandle h) {
        if (precision == VDI_MG_MIXED) {
            VDI_CUDA(cudaMemsetAsync(z32[0], 0, sizeof(float) * size(0), s));
            VDI_TRY(vcycle32(s));
            add_f32_to_f64<<<nblk(size(0)), 256, 0, s>>>(z, z32[0], int(size(0)));
            VDI_TRY(enqueue_resid32(s, b, z, 1, use_cond, h));
        } else {
            VDI_TRY(vcycle64(s, b, z));
            VDI_TRY(enqueue_resid_norm(s, b, z, 1, use_cond, h));
        }
        return VDI_OK;
    }

    int enqueue_first_check(cudaStream_t s, const double* b, const double* z, int precision, int use_cond,
                            cudaGraphConditionalHandle h) {
        if (precision == VDI_MG_MIXED) return enqueue_resid32(s, b, z, 0, use_cond, h);
        return enqueue_resid_norm(s, b, z, 0, use_cond, h);
    }

    int set_ctl_params(cudaStream_t s, double rt, int mx) {
        rtol = rt;
        max_it = mx;
        // rtol and max_it sit at fixed offsets; write them with one copy
        struct P { double rtol; int it; int max_it; } p{rt, 0, mx};
        static_assert(offsetof(SolveCtl, rtol) + sizeof(double) == offsetof(SolveCtl, it), "layout");
        VDI_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(ctl) + offsetof(SolveCtl, rtol), &p,
                                 sizeof(double) + 2 * sizeof(int), cudaMemcpyHostToDevice, s));
        VDI_CUDA(cudaStreamSynchronize(s));
        return VDI_OK;
    }
};

int mg_create(int kind, int m, int n, double c1, double c2, int x_sym, MG** out) {
    if (!out || m < 2 || n < 2 || kind < 0 || kind > 3) {
        set_error("mg_create: invalid arguments");
        return VDI_ERR_INVALID_ARGUMENT;
    }
    MG* g = new MG();
    g->kind = kind; g->m = m; g->n = n; g->c1 = c1; g->c2 = c2; g->x_sym = x_sym;
    int st = g->build_levels();
    if (st == VDI_OK) st = g->alloc();
    if (st != VDI_OK) {
        delete g;
        return st;
    }
    *out = g;
    return VDI_OK;
}

void mg_destroy(MG* mg) { delete mg; }

int mg_set_visc(MG* mg, double vfx, double vfy) {
    if (mg->kind != VDI_MG_VISC_U && mg->kind != VDI_MG_VISC_V) return VDI_ERR_INVALID_ARGUMENT;
    mg->c1 = vfx;
    mg->c2 = vfy;
    double kx = vfx, ky = vfy;
    for (auto& L : mg->lv) {
        mg->fill_cc(L, kx, ky);
        kx *= 0.25; ky *= 0.25;
    }
    return VDI_OK;
}

SolveCtl* mg_ctl(MG* mg) { return mg->ctl; }
int mg_kind(const MG* mg) { return mg->kind; }
int mg_fine_size(const MG* mg) { return int(mg->size(0)); }

int mg_configure(MG* mg, double rtol, int max_it) {
    mg->rtol = rtol;
    mg->max_it = max_it;
    return mg->set_ctl_params(0, rtol, max_it);
}

int mg_solve(MG* mg, cudaStream_t s, const double* b, double* z, double rtol, int max_it, int precision,
             int* vcycles, double* rel_res) {
    if (rtol != mg->rtol || max_it != mg->max_it) VDI_TRY(mg->set_ctl_params(s, rtol, max_it));
    VDI_TRY(mg->enqueue_begin(s, b, z));
    VDI_TRY(mg->enqueue_first_check(s, b, z, precision, 0, 0));
    SolveCtl h{};
    while (true) {
        VDI_CUDA(cudaMemcpyAsync(&h, mg->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, s));
        VDI_CUDA(cudaStreamSynchronize(s));
        if (h.done) break;
        VDI_TRY(mg->enqueue_body(s, b, z, precision, 0, 0));
    }
    if (vcycles) *vcycles = h.it;
    if (rel_res) *rel_res = h.bnorm2 > 0 ? std::sqrt(h.rnorm2 / h.bnorm2) : 0.;
    if (h.status & DEV_NONFINITE) {
        set_error("multigrid: non-finite residual");
        return VDI_ERR_NONFINITE;
    }
    if (h.status & DEV_MG_NOT_CONVERGED) {
        set_error("multigrid: %d V-cycles without reaching rtol %.3g (rel. residual %.3g)", h.it, rtol,
                  h.bnorm2 > 0 ? std::sqrt(h.rnorm2 / h.bnorm2) : 0.);
        return VDI_ERR_MG_NOT_CONVERGED;
    }
    return VDI_OK;
}

int mg_solve_device(MG* mg, cudaStream_t s, const double* b, double* z, int precision) {
    // Without a graph, loop control needs the host; this entry point records
    // the conditional-node loop when s is capturing and otherwise falls back
    // to the host-driven loop.
    cudaStreamCaptureStatus cs;
    VDI_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusActive) return mg_record_graph_solve(mg, s, b, z, precision);
    return mg_solve(mg, s, b, z, mg->rtol, mg->max_it, precision, nullptr, nullptr);
}

int mg_record_graph_solve(MG* mg, cudaStream_t s, const double* b, double* z, int precision) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    VDI_TRY(mg->enqueue_begin(s, b, z));
    VDI_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &ndeps));
    if (cs != cudaStreamCaptureStatusActive) return VDI_ERR_NOT_READY;
    cudaGraphConditionalHandle h;
    VDI_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    VDI_TRY(mg->enqueue_first_check(s, b, z, precision, 1, h));
    VDI_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    VDI_CUDA(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    VDI_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    cudaStream_t bs;
    VDI_CUDA(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) {
        cudaStreamDestroy(bs);
        VDI_CUDA(e);
    }
    int st = mg->enqueue_body(bs, b, z, precision, 1, h);
    cudaGraph_t bodyOut;
    e = cudaStreamEndCapture(bs, &bodyOut);
    cudaStreamDestroy(bs);
    if (st != VDI_OK) return st;
    VDI_CUDA(e);
    return VDI_OK;
}

int mg_v_cycle(MG* mg, cudaStream_t s, const double* b, double* z) { return mg->vcycle64(s, b, z); }

int mg_residual(MG* mg, cudaStream_t s, const double* b, const double* z, double* r, double* norm) {
    double* d_out;
    VDI_CUDA(cudaMallocAsync(&d_out, sizeof(double), s));
    int nb = std::min(mg->norm_blocks(), 4 * 148);
    if (mg->kind == VDI_MG_FEM)
        resid_norm_plain<double><<<nb, 256, 0, s>>>(mg->kind, CCc<double>{}, mg->femc<double>(0), z, b, r, mg->rd,
                                                    d_out);
    else
        resid_norm_plain<double><<<nb, 256, 0, s>>>(mg->kind, mg->ccc<double>(0), FEMc<double>{}, z, b, r, mg->rd,
                                                    d_out);
    VDI_CUDA(cudaGetLastError());
    double hn = 0;
    VDI_CUDA(cudaMemcpyAsync(&hn, d_out, sizeof(double), cudaMemcpyDeviceToHost, s));
    VDI_CUDA(cudaFreeAsync(d_out, s));
    VDI_CUDA(cudaStreamSynchronize(s));
    if (norm) *norm = hn;
    return VDI_OK;
}

int mg_apply(MG* mg, cudaStream_t s, const double* z, double* y) {
    long N = mg->size(0);
    if (mg->kind == VDI_MG_FEM)
        fem_apply<double><<<nblk(N), 256, 0, s>>>(mg->femc<double>(0), z, y);
    else
        cc_apply<double><<<nblk(N), 256, 0, s>>>(mg->ccc<double>(0), z, y);
    VDI_CUDA(cudaGetLastError());
    return VDI_OK;
}

}  // namespace vdi
