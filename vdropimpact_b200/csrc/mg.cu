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
// Each level of a V-cycle above the shared-memory threshold is two launches:
//   PRE : nu1 Gauss-Seidel sweeps, residual, restriction to the coarse source
//   POST: prolongation of the coarse correction, nu2 sweeps, and on the finest
//         level the residual norm and the convergence decision
// Both work on a shared-memory tile whose halo shrinks by one ring per colour
// phase, so a tile computes exactly the values the neighbouring tiles compute
// for the same points. The remaining coarse levels run in one CTA, entirely in
// shared memory. Solves end when ||b-Az||_2 <= rtol*||b||_2. FP32 V-cycles
// inside FP64 iterative refinement use the same kernels with T = float.
#include "vdi_internal.hh"

#include <cudaTypedefs.h>

#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <mutex>
#include <type_traits>

namespace vdi {

static constexpr int MAXLEV = 16;
static constexpr int CTA_THREADS = 1024;
static constexpr size_t CTA_SMEM_LIMIT = 200 * 1024;
static constexpr int MAX_PARTIALS = 8192;
static constexpr int DIRECT_MAX = 256;
// A FEM hierarchy whose first CTA-resident level has more than DIRECT_MAX but
// at most GDIRECT_MAX unknowns solves that level exactly with a dense
// inverse applied by the whole GPU, in place of the single-CTA cycle.
static constexpr int GDIRECT_MAX = 3072;
// A hierarchy whose operator is separable solves its first level of at most
// FAST_MAX unknowns exactly by cosine transforms in x and tridiagonal solves
// in y (mg_fast.cuh), in place of every coarser level.
static constexpr long FAST_MAX = 40000;   // a 75 MB FP64 inverse at most

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
    const int nb = gridDim.x * gridDim.y;
    const int bid = blockIdx.x + gridDim.x * blockIdx.y;
    if (threadIdx.x == 0) {
        rd.partials[bid] = blocksum;
        __threadfence();
        unsigned t = atomicAdd(rd.counter, 1u);
        last = (t == unsigned(nb - 1));
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double s = 0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) s += __ldcg(rd.partials + k);
    s = block_sum(s);
    if (threadIdx.x == 0) {
        *total = s;
        *rd.counter = 0;
    }
    return true;
}

/** grid_sum of two values at once: partials k and nb + k (at most half of
 * the partials array in blocks). */
__device__ bool grid_sum2(double s1, double s2, Reduce rd, double* t1, double* t2) {
    __shared__ int last;
    const int nb = gridDim.x * gridDim.y;
    const int bid = blockIdx.x + gridDim.x * blockIdx.y;
    if (threadIdx.x == 0) {
        rd.partials[bid] = s1;
        rd.partials[nb + bid] = s2;
        __threadfence();
        unsigned t = atomicAdd(rd.counter, 1u);
        last = (t == unsigned(nb - 1));
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double a = 0, b = 0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        a += __ldcg(rd.partials + k);
        b += __ldcg(rd.partials + nb + k);
    }
    a = block_sum(a);
    __syncthreads();
    b = block_sum(b);
    if (threadIdx.x == 0) {
        *t1 = a;
        *t2 = b;
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
    // a failure recorded during the V-cycle (a tile kernel's copy that did
    // not arrive) ends the solve too
    if (ctl->status & (DEV_MG_NOT_CONVERGED | DEV_NONFINITE)) cont = 0;
    if (ctl->status) {
        ctl->sticky |= ctl->status;
        if (ctl->err_out) atomicOr(ctl->err_out, ctl->status);
    }
    if (!cont) {
        ctl->done = 1;
        ctl->solves += 1;
        ctl->vcycles += ctl->it;
        ctl->last_rel = ctl->bnorm2 > 0 ? sqrt(r2 / ctl->bnorm2) : 0.;
    }
    if (use_cond) cudaGraphSetConditional(h, cont);
}

// ------------------------------------------------------- operators
template <typename T>
struct CCc {
    int m, n;
    T ox, oy;          // off-diagonal couplings of A
    T d[3][3];         // diagonal by (x class, y class): 0 first, 1 interior, 2 last
    T invd[3][3];
    signed char gL, gR, gD, gU;
};

template <typename T>
struct FEMc {
    int M, N;
    T fm, fey, hey, fex, hex, fc;
    T d[3][3], invd[3][3];
};

__device__ __forceinline__ int cls(int i, int m) { return i == 0 ? 0 : (i == m - 1 ? 2 : 1); }

/** a[x][y] of a kernel-parameter table. FP32 selects the entry explicitly:
 * indexing the parameter array with computed indices would copy it to the
 * stack; FP64 indexes it (the selections would cost registers it lacks). */
template <typename T>
__device__ __forceinline__ T pick3(const T (&a)[3][3], int x, int y) {
    if constexpr (sizeof(T) == 8) {
        return a[x][y];
    } else {
        const T r0 = y == 0 ? a[0][0] : (y == 1 ? a[0][1] : a[0][2]);
        const T r1 = y == 0 ? a[1][0] : (y == 1 ? a[1][1] : a[1][2]);
        const T r2 = y == 0 ? a[2][0] : (y == 1 ? a[2][1] : a[2][2]);
        return x == 0 ? r0 : (x == 1 ? r1 : r2);
    }
}

/** Off-diagonal part of A z at (i,j); w points at z(i,j) in an array of
 * row pitch P. Neighbours outside the grid do not contribute, as in mul_a
 * of mgs_mac.hh:39-45 and visco_impl.hh:40-46. */
template <typename T>
__device__ __forceinline__ T cc_off(const CCc<T>& c, const T* w, int P, int i, int j) {
    T xs = (i > 0 ? w[-1] : T(0)) + (i < c.m - 1 ? w[1] : T(0));
    T ys = (j > 0 ? w[-P] : T(0)) + (j < c.n - 1 ? w[P] : T(0));
    return c.ox * xs + c.oy * ys;
}

/** mul_a of mgs_fem.cc:32-53 at (i,j); w points at z(i,j), row pitch P. */
template <typename T>
__device__ __forceinline__ T fem_off(const FEMc<T>& c, const T* w, int P, int i, int j) {
    if (j == 0) return T(0);
    const T* wm = w - P;
    const int M = c.M;
    if (j == c.N - 1) {
        if (i == 0) return c.fc * wm[1] + c.hey * (*wm) + c.hex * w[1];
        if (i == M - 1) return c.fc * wm[-1] + c.hey * (*wm) + c.hex * w[-1];
        return c.fc * (wm[-1] + wm[1]) + c.fey * (*wm) + c.hex * (w[-1] + w[1]);
    }
    if (i == 0) return c.fc * (wm[1] + w[P + 1]) + c.hey * (*wm + w[P]) + c.fex * w[1];
    if (i == M - 1) return c.fc * (wm[-1] + w[P - 1]) + c.hey * (*wm + w[P]) + c.fex * w[-1];
    return c.fc * (wm[-1] + wm[1] + w[P - 1] + w[P + 1]) + c.fey * (*wm + w[P]) + c.fex * (w[-1] + w[1]);
}

template <typename T>
__device__ __forceinline__ T op_off(const CCc<T>& c, const T* w, int P, int i, int j) { return cc_off(c, w, P, i, j); }
template <typename T>
__device__ __forceinline__ T op_off(const FEMc<T>& c, const T* w, int P, int i, int j) { return fem_off(c, w, P, i, j); }
template <typename T>
__device__ __forceinline__ int op_m(const CCc<T>& c) { return c.m; }
template <typename T>
__device__ __forceinline__ int op_n(const CCc<T>& c) { return c.n; }
template <typename T>
__device__ __forceinline__ int op_m(const FEMc<T>& c) { return c.M; }
template <typename T>
__device__ __forceinline__ int op_n(const FEMc<T>& c) { return c.N; }

template <class OP, typename T>
__device__ __forceinline__ T op_resid(const OP& c, const T* w, T bv, int P, int i, int j) {
    return bv - pick3(c.d, cls(i, op_m(c)), cls(j, op_n(c))) * (*w) - op_off(c, w, P, i, j);
}
template <class OP, typename T>
__device__ __forceinline__ T op_relaxed(const OP& c, const T* w, T bv, int P, int i, int j) {
    return (bv - op_off(c, w, P, i, j)) * pick3(c.invd, cls(i, op_m(c)), cls(j, op_n(c)));
}

/** Bilinear cell-centred prolongation of the coarse correction to fine cell
 * (i,j) from coarse row r0 = J = j/2 and its neighbour row r1 = J +- 1 (yo:
 * that row is outside the grid, gy its ghost factor); ghost values are
 * g * (boundary value) on each side. */
template <typename T, typename RT>
__device__ __forceinline__ T cc_interp_r(const CCc<T>& f, const RT* r0, const RT* r1, bool yo, T gy, int i) {
    const int mc = f.m >> 1;
    int I = i >> 1;
    int sx = (i & 1) ? 1 : -1;
    int Ix = I + sx;
    bool xo = Ix < 0 || Ix >= mc;
    T gx = T(sx < 0 ? f.gL : f.gR);
    T c00 = T(r0[I]);
    T c10 = xo ? gx * c00 : T(r0[Ix]);
    T c01 = yo ? gy * c00 : T(r1[I]);
    T c11;
    if (xo && yo) c11 = gx * gy * c00;
    else if (xo) c11 = gx * c01;
    else if (yo) c11 = gy * c10;
    else c11 = T(r1[Ix]);
    return T(0.5625) * c00 + T(0.1875) * (c10 + c01) + T(0.0625) * c11;
}
/** The same with row(J) giving coarse row J (indexable by coarse column). */
template <typename T, class ROW>
__device__ __forceinline__ T cc_interp_rows(const CCc<T>& f, ROW row, int i, int j) {
    const int nc = f.n >> 1;
    const int J = j >> 1, sy = (j & 1) ? 1 : -1, Jy = J + sy;
    const bool yo = Jy < 0 || Jy >= nc;
    const T gy = T(sy < 0 ? f.gD : f.gU);
    return cc_interp_r(f, row(J), yo ? row(J) : row(Jy), yo, gy, i);
}
template <typename T, typename TC>
__device__ __forceinline__ T cc_interp(const CCc<T>& f, const TC* zc, int i, int j) {
    const int mc = f.m >> 1;
    return cc_interp_rows(f, [&](int J) { return zc + mc * J; }, i, j);
}

/** Bilinear prolongation of node-centred corrections to fine node (i,j);
 * row(J) gives coarse node row J (indexable by the coarse column). */
template <typename T, class ROW>
__device__ __forceinline__ T fem_interp_rows(const FEMc<T>& f, ROW row, int i, int j) {
    if (j == 0) return T(0);
    int I = i >> 1, J = j >> 1;
    bool ox = i & 1, oy = j & 1;
    const auto* r0 = row(J);
    T c00 = T(r0[I]);
    if (!ox && !oy) return c00;
    if (ox && !oy) return T(0.5) * (c00 + T(r0[I + 1]));
    const auto* r1 = row(J + 1);
    if (!ox && oy) return T(0.5) * (c00 + T(r1[I]));
    return T(0.25) * (c00 + T(r0[I + 1]) + T(r1[I]) + T(r1[I + 1]));
}
template <typename T, typename TC>
__device__ __forceinline__ T fem_interp(const FEMc<T>& f, const TC* zc, int i, int j) {
    const int Mc = (f.M - 1) / 2 + 1;
    return fem_interp_rows(f, [&](int J) { return zc + Mc * J; }, i, j);
}

/** P^T r at coarse node (I,J) from a residual array with origin (ox,oy) and
 * pitch P; zero on the Dirichlet bottom row. */
/** P^T of the bilinear prolongation at coarse node (I, J), fine residuals
 * read through at(i, j). */
template <typename T, typename F>
__device__ __forceinline__ T fem_restrict_by(int M, int N, F at, int I, int J) {
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
            s += wx * wy * at(i, j);
        }
    }
    return s;
}

template <typename T>
__device__ __forceinline__ T fem_restrict_at(int M, int N, const T* r, int P, int ox, int oy, int I, int J) {
    return fem_restrict_by<T>(M, N, [&](int i, int j) { return r[(i - ox) + P * (j - oy)]; }, I, J);
}

// ------------------------------------------------------- fused tile kernels
template <typename T, typename TC = T>
struct TileArgs {
    const T* zin;      // iterate read (PRE: unless zero_init; POST: before the correction)
    T* zout;           // iterate written; never the array zin points to, because
                       // neighbouring tiles read zin as their halo concurrently
    const T* b;
    TC* bc;            // PRE: coarse source out (the coarse levels' precision)
    const TC* zc;      // POST: coarse correction in
    int zero_init;     // PRE: z starts from zero (coarse levels)
    int norm;          // POST: residual norm + decision
    Reduce rd;
    SolveCtl* ctl;
    int use_cond;
    cudaGraphConditionalHandle h;
};

template <typename T, int NS>
struct CCTile {
    static constexpr int CW = 64, CH = 64, KW = CW / 2;
    static constexpr int K = 2 * NS, ZH = K + 1;
    static constexpr int TX = CW - 2 * ZH, TY = CH - 2 * ZH;
    static constexpr int NT = 512, NW = NT / 32;
    // the two colour arrays of z (and of b) sit 64 bytes off each other's
    // bank alignment: a warp over consecutive columns alternates between
    // them, and its half-warps then fall in different banks
    static constexpr int CSTR = CH * KW + 64 / int(sizeof(T));
    static constexpr size_t smem = size_t(4) * CSTR * sizeof(T);
};

/** MODE 0: NS sweeps from zin (or zero), residual, restriction to bc (skipped
 * when bc is null). MODE 1: zin + prolonged zc, NS sweeps, and optionally the
 * residual norm with the solve decision. Both write zout. */
/** The colour phases of a cell-centred window held in Z/B (split by
 * colour); par0 is the colour parity of the window origin (zx, zy). */
template <typename T, int MODE, int NS>
__device__ __forceinline__ void cc_window_phases(const CCc<T>& c, T* Z, const T* B, int par0, bool inner, int zx,
                                                 int zy) {
    using G = CCTile<T, NS>;
    constexpr int CW = G::CW, CH = G::CH, KW = G::KW, K = G::K;
    constexpr int NW = G::NW, RPW = CH / NW;
    const int m = c.m, n = c.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int ph = 0; ph < K; ph++) {
        const int color = MODE == 1 ? ((ph & 1) ^ 1) : (ph & 1);
        T* Zc = Z + color * G::CSTR;
        const T* Zo = Z + (color ^ 1) * G::CSTR;
        const T* Bc = B + color * G::CSTR;
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            const int jj = warp + q * NW;
            // phase ph can only be exact at ph+1 or more cells from the
            // window's edge (its neighbours nearer the edge are stale)
            if (jj < ph + 1 || jj > CH - 2 - ph) continue;
            const int p = (color ^ par0 ^ jj) & 1;
            const int ii = 2 * lane + p;
            if (ii < ph + 1 || ii > CW - 2 - ph) continue;
            const T* zo = Zo + jj * KW;
            const T l = zo[lane - 1 + p], r = zo[lane + p];
            const T d = Zo[(jj - 1) * KW + lane], u = Zo[(jj + 1) * KW + lane];
            T* w = Zc + jj * KW + lane;
            if (inner) {
                *w = (Bc[jj * KW + lane] - (c.ox * (l + r) + c.oy * (d + u))) * c.invd[1][1];
            } else {
                const int i = zx + ii, j = zy + jj;
                if (unsigned(i) >= unsigned(m) || unsigned(j) >= unsigned(n)) continue;
                T xs = (i > 0 ? l : T(0)) + (i < m - 1 ? r : T(0));
                T ys = (j > 0 ? d : T(0)) + (j < n - 1 ? u : T(0));
                *w = (Bc[jj * KW + lane] - (c.ox * xs + c.oy * ys)) * pick3(c.invd, cls(i, m), cls(j, n));
            }
        }
        __syncthreads();
    }
}

/** The end of a window: its interior written to zout, and (PRE) the
 * restricted residual written to bc or (POST with norm) the window's sum of
 * squared residuals returned. */
template <typename T, int MODE, int NS, typename TC>
__device__ __forceinline__ double cc_window_epilogue(const CCc<T>& c, const TileArgs<T, TC>& a, const T* Z,
                                                    const T* B, int par0, int x0, int y0, int zx, int zy) {
    using G = CCTile<T, NS>;
    constexpr int CH = G::CH, KW = G::KW, ZH = G::ZH, TX = G::TX, TY = G::TY;
    constexpr int NW = G::NW;
    const int m = c.m, n = c.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    auto zat = [&](int ii, int jj) -> T { return Z[((par0 + ii + jj) & 1) * G::CSTR + jj * KW + (ii >> 1)]; };
    auto resid = [&](int ii, int jj) -> T {
        const int i = zx + ii, j = zy + jj;
        T bv = B[((par0 + ii + jj) & 1) * G::CSTR + jj * KW + (ii >> 1)];
        T xs = (i > 0 ? zat(ii - 1, jj) : T(0)) + (i < m - 1 ? zat(ii + 1, jj) : T(0));
        T ys = (j > 0 ? zat(ii, jj - 1) : T(0)) + (j < n - 1 ? zat(ii, jj + 1) : T(0));
        return bv - pick3(c.d, cls(i, m), cls(j, n)) * zat(ii, jj) - (c.ox * xs + c.oy * ys);
    };
    // interior back to global memory (coalesced by row)
    for (int jj = ZH + warp; jj < ZH + TY; jj += NW) {
        const int j = zy + jj;
        if (j >= n) break;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int ii = ZH + lane + 32 * h;
            const int i = zx + ii;
            if (ii < ZH + TX && i < m) a.zout[i + m * j] = zat(ii, jj);
        }
    }
    double s = 0;
    if (MODE == 0) {
        if (a.bc) {
            const int mc = m >> 1, nc = n >> 1;
            constexpr int CX = TX / 2, CY = TY / 2;
            for (int t = threadIdx.x; t < CX * CY; t += G::NT) {
                const int q = t / CX;
                const int I = x0 / 2 + (t - q * CX), J = y0 / 2 + q;
                if (I >= mc || J >= nc) continue;
                const int ii = 2 * I - zx, jj = 2 * J - zy;
                T r = resid(ii, jj) + resid(ii + 1, jj) + resid(ii, jj + 1) + resid(ii + 1, jj + 1);
                a.bc[I + mc * J] = TC(T(0.25) * r);
            }
        }
    } else if (a.norm) {
        // a warp takes the row's cells of one colour (every other column),
        // so each read of the residual is consecutive words of one colour
        // array; consecutive columns alternate arrays whose words share banks
        static_assert(TX / 2 <= 32 && TX % 2 == 0, "one warp per colour row");
        for (int jj = ZH + warp; jj < ZH + TY; jj += NW) {
            const int j = zy + jj;
            if (j >= n) break;
#pragma unroll
            for (int ci = 0; ci < 2; ci++) {
                const int ii = ZH + ci + 2 * lane;
                if (ii < ZH + TX && zx + ii < m) {
                    double r = double(resid(ii, jj));
                    s += r * r;
                }
            }
        }
    }
    return s;
}

template <typename T, int MODE, int NS, typename TC = T>
__global__ void __launch_bounds__(CCTile<T, NS>::NT) cc_tile(CCc<T> c, TileArgs<T, TC> a) {
    using G = CCTile<T, NS>;
    constexpr int CW = G::CW, CH = G::CH, KW = G::KW, ZH = G::ZH, TX = G::TX, TY = G::TY;
    constexpr int NW = G::NW, RPW = CH / NW;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    T* Z = reinterpret_cast<T*>(sm_raw);
    T* B = Z + 2 * G::CSTR;
    const int m = c.m, n = c.n;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int zx = x0 - ZH, zy = y0 - ZH;
    const int par0 = (zx + zy) & 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool inner = zx >= 0 && zy >= 0 && zx + CW <= m && zy + CH <= n;
    const bool read_z = MODE == 1 || !a.zero_init;
    // ---- load: every load of the thread issued before the shared stores
    {
        T zv[RPW][2], bv[RPW][2];
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            int jj = warp + q * NW, j = zy + jj;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int i = zx + lane + 32 * h;
                bool in = unsigned(i) < unsigned(m) && unsigned(j) < unsigned(n);
                zv[q][h] = (in && read_z) ? a.zin[i + m * j] : T(0);
                bv[q][h] = in ? a.b[i + m * j] : T(0);
            }
        }
        if constexpr (MODE == 1) {
            // POST: the coarse correction of the window (coarse columns and
            // rows (zx>>1)-1 .. ((zx+63)>>1)+1, 35 of each since the window
            // origin is odd) staged in shared memory, then prolonged from there
            constexpr int CC = CW / 2 + 3;
            static_assert(CC == CH / 2 + 3, "square window");
            __shared__ TC cwin[CC * CC];
            const int mc = m >> 1, nc = n >> 1, I0 = (zx >> 1) - 1, J0 = (zy >> 1) - 1;
            constexpr int PER = (CC * CC + G::NT - 1) / G::NT;
            TC cv[PER];
#pragma unroll
            for (int u = 0; u < PER; u++) {
                const int k = threadIdx.x + u * G::NT, Jl = k / CC, I = I0 + (k - Jl * CC), J = J0 + Jl;
                cv[u] = (k < CC * CC && unsigned(I) < unsigned(mc) && unsigned(J) < unsigned(nc)) ? a.zc[I + mc * J]
                                                                                                 : TC(0);
            }
#pragma unroll
            for (int u = 0; u < PER; u++)
                if (threadIdx.x + u * G::NT < CC * CC) cwin[threadIdx.x + u * G::NT] = cv[u];
            __syncthreads();
            auto row = [&](int J) { return cwin + (J - J0) * CC - I0; };
#pragma unroll
            for (int q = 0; q < RPW; q++) {
                const int j = zy + warp + q * NW;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int i = zx + lane + 32 * h;
                    if (unsigned(i) < unsigned(m) && unsigned(j) < unsigned(n)) zv[q][h] += cc_interp_rows(c, row, i, j);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            int jj = warp + q * NW;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int ii = lane + 32 * h;
                int col = (par0 + ii + jj) & 1;
                Z[col * G::CSTR + jj * KW + (ii >> 1)] = zv[q][h];
                B[col * G::CSTR + jj * KW + (ii >> 1)] = bv[q][h];
            }
        }
    }
    __syncthreads();
    cc_window_phases<T, MODE, NS>(c, Z, B, par0, inner, zx, zy);
    double s = cc_window_epilogue<T, MODE, NS, TC>(c, a, Z, B, par0, x0, y0, zx, zy);
    if (MODE == 1 && a.norm) {
        s = block_sum(s);
        double total;
        if (grid_sum(s, a.rd, &total) && threadIdx.x == 0) solve_decide(a.ctl, total, 1, a.use_cond, a.h);
    }
}

// ---------------------------------------- register-blocked cell-centred tile
// The same window computation as cc_tile (a 64 x 64 window, its halo
// shrinking one ring per colour phase, the same update and residual
// arithmetic), laid out so the phases touch no shared memory in the inner
// loop: thread (warp w, lane t) holds columns 2t, 2t+1 and rows 8w..8w+7 of
// the window in registers. A red-black update then finds its vertical
// neighbours in its own registers, one horizontal neighbour in its own other
// column and the other in the adjacent lane (a shuffle); only each warp's
// first and last row cross warps, through a small double-buffered shared
// array, once per phase. The window origin is even, so a thread's 2 x 2
// blocks are exactly the coarse cells: restriction and the prolongation's
// coarse neighbourhood stay in registers too.
template <typename T>
struct CCReg {
    static constexpr int R = 8;                 // rows per thread
    static constexpr int NWARP = 8;
    static constexpr int NT = 32 * NWARP;
    static constexpr int CW = 64, CH = R * NWARP;
    static constexpr int K = 4;                 // colour phases: two red-black sweeps
    static constexpr int ZH = 6;                // K + 1 rings, rounded up to even
    static constexpr int TX = CW - 2 * ZH, TY = CH - 2 * ZH;
};


template <typename T>
__device__ __forceinline__ T shfl_up1(T v) { return __shfl_up_sync(0xffffffffu, v, 1); }
template <typename T>
__device__ __forceinline__ T shfl_dn1(T v) { return __shfl_down_sync(0xffffffffu, v, 1); }

/** MODE 0: NS = 2 sweeps from zin (or zero), residual, restriction to bc
 * (skipped when bc is null). MODE 1: zin + prolonged zc, 2 sweeps, and
 * optionally the residual norm with the solve decision. Both write zout. */
/** One window of the register-blocked cell-centred tile (window origin zx,
 * zy, both even) from z and b already in registers: the prolongation of the
 * coarse correction (MODE 1), the colour phases, the interior written to
 * zout and, when asked, the restriction to bc (MODE 0) or the thread's sum
 * of squared residuals over the interior, returned (MODE 1 with norm). Every
 * thread of the CTA must call it: the phases synchronise the CTA. */
template <typename T, int MODE, typename TC>
__device__ __forceinline__ double cc_rwin(const CCc<T>& c, const TileArgs<T, TC>& a, T (&z)[CCReg<T>::R][2],
                                          const T (&b)[CCReg<T>::R][2], int zx, int zy,
                                          T (*edge)[2][CCReg<T>::NWARP][CCReg<T>::CW]) {
    using G = CCReg<T>;
    constexpr int R = G::R, CW = G::CW, CH = G::CH, K = G::K, ZH = G::ZH, NWARP = G::NWARP;
    const int m = c.m, n = c.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i0 = zx + 2 * lane, j0 = zy + warp * R;
    const bool vec = (m & 1) == 0 && (reinterpret_cast<uintptr_t>(a.zout) & (2 * sizeof(T) - 1)) == 0;
    using T2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    const bool colin = i0 >= 0 && i0 + 1 < m;
    if constexpr (MODE == 1) {
        // prolongation: coarse cell I = i0/2 covers this thread's columns;
        // fine rows j0..j0+7 use coarse rows J0-1 .. J0+4
        const int mc = m >> 1, nc = n >> 1, I = i0 >> 1, J0 = j0 >> 1;
        constexpr int CR = R / 2 + 2;
        T cm[CR], cc[CR], cp[CR];
#pragma unroll
        for (int q = 0; q < CR; q++) {
            const int J = J0 - 1 + q;
            const bool rin = unsigned(J) < unsigned(nc);
            cc[q] = (rin && unsigned(I) < unsigned(mc)) ? T(a.zc[I + long(mc) * J]) : T(0);
            cm[q] = shfl_up1(cc[q]);
            cp[q] = shfl_dn1(cc[q]);
            if (lane == 0) cm[q] = (rin && unsigned(I - 1) < unsigned(mc)) ? T(a.zc[I - 1 + long(mc) * J]) : T(0);
            if (lane == 31) cp[q] = (rin && unsigned(I + 1) < unsigned(mc)) ? T(a.zc[I + 1 + long(mc) * J]) : T(0);
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int j = j0 + r;
            const int qJ = 1 + r / 2;                  // coarse row J = j >> 1 in the register window
            const int sy = (r & 1) ? 1 : -1;           // j0 is even
            const int Jy = (j >> 1) + sy;
            const bool yo = Jy < 0 || Jy >= nc;
            const T gy = T(sy < 0 ? c.gD : c.gU);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int i = i0 + h;
                if (!(unsigned(i) < unsigned(m) && unsigned(j) < unsigned(n))) continue;
                const int Ix = I + (h ? 1 : -1);
                const bool xo = Ix < 0 || Ix >= mc;
                const T gx = T(h ? c.gR : c.gL);
                const T c00 = cc[qJ];
                const T s0 = h ? cp[qJ] : cm[qJ], s1 = h ? cp[qJ + sy] : cm[qJ + sy];
                const T c10 = xo ? gx * c00 : s0;
                const T c01 = yo ? gy * c00 : cc[qJ + sy];
                T c11;
                if (xo && yo) c11 = gx * gy * c00;
                else if (xo) c11 = gx * c01;
                else if (yo) c11 = gy * c10;
                else c11 = s1;
                z[r][h] += T(0.5625) * c00 + T(0.1875) * (c10 + c01) + T(0.0625) * c11;
            }
        }
    }
    // colour phases: colour (i + j) & 1 = col; in row r the thread's point of
    // that colour is column h = (col + r) & 1 (i0 and j0 are even)
#pragma unroll
    for (int ph = 0; ph < K; ph++) {
        const int col = MODE == 1 ? ((ph & 1) ^ 1) : (ph & 1);
        T(*eb)[NWARP][CW] = edge[ph & 1];
        reinterpret_cast<T2*>(&eb[0][warp][0])[lane] = T2{z[0][0], z[0][1]};
        reinterpret_cast<T2*>(&eb[1][warp][0])[lane] = T2{z[R - 1][0], z[R - 1][1]};
        __syncthreads();
        T below[2], above[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            below[h] = warp > 0 ? eb[1][warp - 1][2 * lane + h] : T(0);
            above[h] = warp < NWARP - 1 ? eb[0][warp + 1][2 * lane + h] : T(0);
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int h = (col + r) & 1;
            const int j = j0 + r, i = i0 + h;
            // left and right neighbours: the thread's other column, and the
            // facing column of the adjacent lane
            T l, rr;
            if (h == 0) {
                l = shfl_up1(z[r][1]);
                rr = z[r][1];
            } else {
                l = z[r][0];
                rr = shfl_dn1(z[r][0]);
            }
            const T d = r > 0 ? z[r > 0 ? r - 1 : 0][h] : below[h];
            const T u = r < R - 1 ? z[r < R - 1 ? r + 1 : R - 1][h] : above[h];
            const int ii = 2 * lane + h, jj = warp * R + r;
            // computed for every row and kept where the point is in the grid
            // and exact in this phase: no branch between the (independent)
            // rows, so their arithmetic interleaves
            const bool upd = ii >= ph + 1 && ii <= CW - 2 - ph && jj >= ph + 1 && jj <= CH - 2 - ph &&
                             unsigned(i) < unsigned(m) && unsigned(j) < unsigned(n);
            const T xs = (i > 0 ? l : T(0)) + (i < m - 1 ? rr : T(0));
            const T ys = (j > 0 ? d : T(0)) + (j < n - 1 ? u : T(0));
            const T zn = (b[r][h] - (c.ox * xs + c.oy * ys)) * pick3(c.invd, cls(i, m), cls(j, n));
            z[r][h] = upd ? zn : z[r][h];
        }
    }
    // interior back to global memory
    const bool lanein = 2 * lane >= ZH && 2 * lane < ZH + G::TX;
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int jj = warp * R + r, j = j0 + r;
        if (!lanein || jj < ZH || jj >= ZH + G::TY || j >= n) continue;
        if (colin && vec) {
            *reinterpret_cast<T2*>(a.zout + i0 + long(m) * j) = T2{z[r][0], z[r][1]};
        } else {
#pragma unroll
            for (int h = 0; h < 2; h++)
                if (i0 + h < m) a.zout[i0 + h + long(m) * j] = z[r][h];
        }
    }
    const bool want_resid = MODE == 0 ? a.bc != nullptr : a.norm != 0;
    if (!want_resid) return 0.;
    // residual of the final iterate at the thread's points (vertical
    // neighbours across warps once more through the shared array)
    {
        T(*eb)[NWARP][CW] = edge[K & 1];
        reinterpret_cast<T2*>(&eb[0][warp][0])[lane] = T2{z[0][0], z[0][1]};
        reinterpret_cast<T2*>(&eb[1][warp][0])[lane] = T2{z[R - 1][0], z[R - 1][1]};
    }
    __syncthreads();
    T below[2], above[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        below[h] = warp > 0 ? edge[K & 1][1][warp - 1][2 * lane + h] : T(0);
        above[h] = warp < NWARP - 1 ? edge[K & 1][0][warp + 1][2 * lane + h] : T(0);
    }
    T res[R][2];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int j = j0 + r;
        const T lft = shfl_up1(z[r][1]), rgt = shfl_dn1(z[r][0]);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int i = i0 + h;
            const T l = h == 0 ? lft : z[r][0];
            const T rr = h == 0 ? z[r][1] : rgt;
            const T d = r > 0 ? z[r > 0 ? r - 1 : 0][h] : below[h];
            const T u = r < R - 1 ? z[r < R - 1 ? r + 1 : R - 1][h] : above[h];
            const int ci = cls(i, m), cj = cls(j, n);
            const T xs = (i > 0 ? l : T(0)) + (i < m - 1 ? rr : T(0));
            const T ys = (j > 0 ? d : T(0)) + (j < n - 1 ? u : T(0));
            res[r][h] = b[r][h] - pick3(c.d, ci, cj) * z[r][h] - (c.ox * xs + c.oy * ys);
        }
    }
    if constexpr (MODE == 0) {
        const int mc = m >> 1, nc = n >> 1, I = i0 >> 1;
#pragma unroll
        for (int k = 0; k < R / 2; k++) {
            const int jj = warp * R + 2 * k, J = (j0 >> 1) + k;
            if (!lanein || jj < ZH || jj >= ZH + G::TY || unsigned(I) >= unsigned(mc) || unsigned(J) >= unsigned(nc))
                continue;
            const T s4 = res[2 * k][0] + res[2 * k][1] + res[2 * k + 1][0] + res[2 * k + 1][1];
            a.bc[I + long(mc) * J] = TC(T(0.25) * s4);
        }
        return 0.;
    } else {
        double s = 0;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int jj = warp * R + r, j = j0 + r;
            if (!lanein || jj < ZH || jj >= ZH + G::TY || j >= n) continue;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                if (i0 + h >= m) continue;
                const double rv = double(res[r][h]);
                s += rv * rv;
            }
        }
        return s;
    }
}

/** The register-blocked tile as one window per CTA, loaded straight from
 * global memory into registers. */
template <typename T, int MODE, typename TC = T, int MINB = 2>
__global__ void __launch_bounds__(CCReg<T>::NT, MINB) cc_rtile(CCc<T> c, TileArgs<T, TC> a) {
    using G = CCReg<T>;
    constexpr int R = G::R, CW = G::CW, ZH = G::ZH, NWARP = G::NWARP;
    const int m = c.m, n = c.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int zx = blockIdx.x * G::TX - ZH, zy = blockIdx.y * G::TY - ZH;
    const int i0 = zx + 2 * lane, j0 = zy + warp * R;
    const bool read_z = MODE == 1 || !a.zero_init;
    const bool vec = (m & 1) == 0 && ((reinterpret_cast<uintptr_t>(a.zin) | reinterpret_cast<uintptr_t>(a.b) |
                                       reinterpret_cast<uintptr_t>(a.zout)) & (2 * sizeof(T) - 1)) == 0;
    using T2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    const bool colin = i0 >= 0 && i0 + 1 < m;
    T z[R][2], b[R][2];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int j = j0 + r;
        const bool rowin = unsigned(j) < unsigned(n);
        if (rowin && colin && vec) {
            const long o = i0 + long(m) * j;
            T2 bv = *reinterpret_cast<const T2*>(a.b + o);
            b[r][0] = bv.x; b[r][1] = bv.y;
            if (read_z) {
                T2 zv = *reinterpret_cast<const T2*>(a.zin + o);
                z[r][0] = zv.x; z[r][1] = zv.y;
            } else {
                z[r][0] = z[r][1] = T(0);
            }
        } else {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int i = i0 + h;
                const bool in = rowin && unsigned(i) < unsigned(m);
                b[r][h] = in ? a.b[i + long(m) * j] : T(0);
                z[r][h] = (in && read_z) ? a.zin[i + long(m) * j] : T(0);
            }
        }
    }
    __shared__ __align__(16) T edge_s[2][2][NWARP][CW];
    const double s = cc_rwin<T, MODE, TC>(c, a, z, b, zx, zy, edge_s);
    if (MODE == 1 && a.norm) {
        const double t = block_sum(s);
        double total;
        if (grid_sum(t, a.rd, &total) && threadIdx.x == 0) solve_decide(a.ctl, total, 1, a.use_cond, a.h);
    }
}

// --------------------------------- persistent, TMA-fed register tile
// The register-blocked window computation in a persistent kernel: one CTA
// per SM walks windows blockIdx.x, blockIdx.x + gridDim.x, ..., and while it
// computes one window, a bulk tensor copy (TMA, plain 2D loads of this GPU's
// own arrays, no multicast) brings the next window's z and b into the other
// half of a two-stage shared-memory ring. Threads take their 2 x 8 blocks from
// the staged window, so the phases run from registers as in cc_rtile.
// FP64 only: a window origin is even, and the copy's x coordinate must be a
// multiple of 16 bytes.
struct PTileStage {
    static constexpr int W = CCReg<double>::CW, H = CCReg<double>::CH;
    static constexpr size_t BYTES = size_t(W) * H * sizeof(double);   // one array of one window
    static constexpr size_t SMEM = 4 * BYTES;                          // z and b, two stages
};

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        :
        : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(dst))), "l"(map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

/** Bounded wait on an mbarrier phase (about 0.5 s of SM clock); false if it
 * gave up. */
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > 1000000000LL) return false;
    }
}

template <int MODE, typename TC>
__global__ void __launch_bounds__(CCReg<double>::NT, 1)
    cc_ptile(CCc<double> c, TileArgs<double, TC> a, const __grid_constant__ CUtensorMap mz,
             const __grid_constant__ CUtensorMap mb, int nwx, int nwin) {
    using G = CCReg<double>;
    constexpr int R = G::R, CW = G::CW, ZH = G::ZH, NWARP = G::NWARP;
    extern __shared__ __align__(1024) unsigned char pt_raw[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ __align__(16) double edge_s[2][2][NWARP][CW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool read_z = MODE == 1 || !a.zero_init;
    const uint32_t tx = uint32_t(read_z ? 2 : 1) * uint32_t(PTileStage::BYTES);
    auto zst = [&](int st) { return reinterpret_cast<double*>(pt_raw + size_t(2 * st) * PTileStage::BYTES); };
    auto bst = [&](int st) { return reinterpret_cast<double*>(pt_raw + size_t(2 * st + 1) * PTileStage::BYTES); };
    auto bar_of = [&](int st) { return static_cast<uint32_t>(__cvta_generic_to_shared(&bars[st])); };
    auto issue = [&](int w, int st) {
        const int zx = (w % nwx) * G::TX - ZH, zy = (w / nwx) * G::TY - ZH;
        mbar_expect(bar_of(st), tx);
        tma_load_2d(bst(st), &mb, zx, zy, bar_of(st));
        if (read_z) tma_load_2d(zst(st), &mz, zx, zy, bar_of(st));
    };
    if (threadIdx.x == 0) {
        for (int st = 0; st < 2; st++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_of(st)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (int(blockIdx.x) < nwin) issue(blockIdx.x, 0);
        if (int(blockIdx.x + gridDim.x) < nwin) issue(blockIdx.x + gridDim.x, 1);
    }
    double s = 0;
    int ok = 1;
    int k = 0;
    int w = blockIdx.x;
    for (; w < nwin; w += gridDim.x, k++) {
        const int st = k & 1;
        ok = mbar_wait_bounded(bar_of(st), uint32_t((k >> 1) & 1)) ? 1 : 0;
        ok = __syncthreads_and(ok);
        if (!ok) break;
        const int zx = (w % nwx) * G::TX - ZH, zy = (w / nwx) * G::TY - ZH;
        double z[R][2], b[R][2];
        const double* zs = zst(st);
        const double* bs = bst(st);
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int o = (warp * R + r) * CW + 2 * lane;
            const double2 bv = *reinterpret_cast<const double2*>(bs + o);
            b[r][0] = bv.x;
            b[r][1] = bv.y;
            if (read_z) {
                const double2 zv = *reinterpret_cast<const double2*>(zs + o);
                z[r][0] = zv.x;
                z[r][1] = zv.y;
            } else {
                z[r][0] = z[r][1] = 0.;
            }
        }
        // every thread has its values: the stage takes the window after next
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0 && w + 2 * int(gridDim.x) < nwin) issue(w + 2 * gridDim.x, st);
        s += cc_rwin<double, MODE, TC>(c, a, z, b, zx, zy, edge_s);
    }
    if (!ok) {
        // a copy did not arrive in time: the solve fails (its control block
        // says so, and the owner's error word when there is one), and the
        // copies that may still be in flight, windows k and k+1, get a
        // bounded wait before the CTA leaves
        if (threadIdx.x == 0) {
            atomicOr(&a.ctl->status, int(DEV_MG_NOT_CONVERGED));
            atomicOr(&a.ctl->sticky, int(DEV_MG_NOT_CONVERGED));
            atomicExch(&a.ctl->tma_timeout, 1);
            if (a.ctl->err_out) atomicOr(a.ctl->err_out, int(DEV_MG_NOT_CONVERGED));
            for (int d = 0; d < 2; d++) {
                const int kk = k + d;
                if (w + d * int(gridDim.x) < nwin) (void)mbar_wait_bounded(bar_of(kk & 1), uint32_t((kk >> 1) & 1));
            }
        }
        __syncthreads();
        // the CTA still joins the norm's grid reduction below, so the solve's
        // decision is made (and, with the failure bit set, ends the solve)
    }
    if (MODE == 1 && a.norm) {
        const double t = block_sum(s);
        double total;
        if (grid_sum(t, a.rd, &total) && threadIdx.x == 0) solve_decide(a.ctl, total, 1, a.use_cond, a.h);
    }
}

// -------------------------------------- four-colour split node-centred tile
// The FEM system's tile: a 64 x 64 window with an even origin, so window point
// (ii,jj) has colour (ii&1, jj&1); each colour lives in its own 32 x 32
// quarter array Q[ci+2cj][jj>>1][ii>>1]. A warp updates one quarter-row with
// 32 consecutive words; all eight neighbours are consecutive words of the
// other quarters. As in the cell-centred tile, every phase updates the whole
// window and the halo (10 rings for 8 colour phases plus the residual ring of
// the restriction) keeps the stale edge out of the interior results.
template <typename T>
struct FEMTile {
    static constexpr int CW = 64, CH = 64, QW = 32, QN = QW * QW;
    static constexpr int K = 8, ZH = 10;
    static constexpr int TX = CW - 2 * ZH, TY = CH - 2 * ZH;
    static constexpr int RW = TX + 2, RH = TY + 2;
    static constexpr int NT = 512, NW = NT / 32;
    // quarters 64 bytes off each other's bank alignment, for the passes in
    // which a warp over consecutive columns alternates between two of them
    static constexpr int QS = QN + 64 / int(sizeof(T));
    static constexpr size_t smem = (size_t(8) * QS + size_t(RW) * RH) * sizeof(T);
};

/** mul_a of mgs_fem.cc:32-53 from neighbour values (dl d dr / l r / ul u ur). */
template <typename T>
__device__ __forceinline__ T fem_off_vals(const FEMc<T>& c, int i, int j, T dl, T d, T dr, T l, T r, T ul, T u,
                                          T ur) {
    if (j == 0) return T(0);
    if (j == c.N - 1) {
        if (i == 0) return c.fc * dr + c.hey * d + c.hex * r;
        if (i == c.M - 1) return c.fc * dl + c.hey * d + c.hex * l;
        return c.fc * (dl + dr) + c.fey * d + c.hex * (l + r);
    }
    if (i == 0) return c.fc * (dr + ur) + c.hey * (d + u) + c.fex * r;
    if (i == c.M - 1) return c.fc * (dl + ul) + c.hey * (d + u) + c.fex * l;
    return c.fc * (dl + dr + ul + ur) + c.fey * (d + u) + c.fex * (l + r);
}

template <typename T, int MODE, typename TC = T>
__global__ void __launch_bounds__(FEMTile<T>::NT) fem_tile(FEMc<T> c, TileArgs<T, TC> a) {
    using G = FEMTile<T>;
    constexpr int QW = G::QW, QN = G::QN, ZH = G::ZH, TX = G::TX, TY = G::TY, K = G::K, NW = G::NW;
    constexpr int CH = G::CH, RW = G::RW, RH = G::RH;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    T* Z = reinterpret_cast<T*>(sm_raw);     // 4 quarters
    T* B = Z + 4 * G::QS;                    // 4 quarters
    T* R = B + 4 * G::QS;                    // residual ring array (PRE)
    const int M = c.M, N = c.N;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int zx = x0 - ZH, zy = y0 - ZH;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool inner = zx >= 0 && zy >= 0 && zx + G::CW <= M && zy + CH <= N && zy > 0;
    const bool read_z = MODE == 1 || !a.zero_init;
    auto qidx = [](int ii, int jj) { return ((ii & 1) + 2 * (jj & 1)) * G::QS + (jj >> 1) * QW + (ii >> 1); };
    {
        constexpr int RPW = CH / NW;
        T zv[RPW][2], bv[RPW][2];
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            int jj = warp + q * NW, j = zy + jj;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int i = zx + lane + 32 * h;
                bool in = unsigned(i) < unsigned(M) && unsigned(j) < unsigned(N);
                zv[q][h] = (in && read_z) ? a.zin[i + M * j] : T(0);
                bv[q][h] = in ? a.b[i + M * j] : T(0);
            }
        }
        if constexpr (MODE == 1) {
            // POST: the coarse correction of the window (coarse nodes
            // zx/2 .. zx/2+32 by zy/2 .. zy/2+32; the window origin is even)
            // staged in shared memory, then prolonged from there
            constexpr int CC = G::CW / 2 + 1;
            static_assert(CC == CH / 2 + 1, "square window");
            __shared__ TC cwin[CC * CC];
            const int Mc = (M - 1) / 2 + 1, Nc = (N - 1) / 2 + 1, I0 = zx >> 1, J0 = zy >> 1;
            constexpr int PER = (CC * CC + G::NT - 1) / G::NT;
            TC cv[PER];
#pragma unroll
            for (int u = 0; u < PER; u++) {
                const int k = threadIdx.x + u * G::NT, Jl = k / CC, I = I0 + (k - Jl * CC), J = J0 + Jl;
                cv[u] = (k < CC * CC && unsigned(I) < unsigned(Mc) && unsigned(J) < unsigned(Nc)) ? a.zc[I + Mc * J]
                                                                                                 : TC(0);
            }
#pragma unroll
            for (int u = 0; u < PER; u++)
                if (threadIdx.x + u * G::NT < CC * CC) cwin[threadIdx.x + u * G::NT] = cv[u];
            __syncthreads();
            auto row = [&](int J) { return cwin + (J - J0) * CC - I0; };
#pragma unroll
            for (int q = 0; q < RPW; q++) {
                const int j = zy + warp + q * NW;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int i = zx + lane + 32 * h;
                    if (unsigned(i) < unsigned(M) && unsigned(j) < unsigned(N)) zv[q][h] += fem_interp_rows(c, row, i, j);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            int jj = warp + q * NW;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int ii = lane + 32 * h;
                Z[qidx(ii, jj)] = zv[q][h];
                B[qidx(ii, jj)] = bv[q][h];
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int ph = 0; ph < K; ph++) {
        const int color = MODE == 1 ? 3 - (ph & 3) : (ph & 3);
        const int ci = color & 1, cj = color >> 1;
        T* Zc = Z + color * G::QS;
        const T* Zx = Z + (color ^ 1) * G::QS;   // (1-ci, cj): left/right
        const T* Zy = Z + (color ^ 2) * G::QS;   // (ci, 1-cj): down/up
        const T* Zd = Z + (color ^ 3) * G::QS;   // (1-ci, 1-cj): diagonals
        const T* Bc = B + color * G::QS;
#pragma unroll
        for (int q = 0; q < QW / NW; q++) {
            const int jr = warp + q * NW, ir = lane;
            const int ii = 2 * ir + ci, jj = 2 * jr + cj;
            // phase ph can only be exact at ph+1 or more cells from the
            // window's edge (its neighbours nearer the edge are stale)
            if (ii < ph + 1 || ii > G::CW - 2 - ph || jj < ph + 1 || jj > CH - 2 - ph) continue;
            const int xl = ir - 1 + ci, xr = ir + ci, yd = jr - 1 + cj, yu = jr + cj;
            const T l = Zx[jr * QW + xl], r = Zx[jr * QW + xr];
            const T d = Zy[yd * QW + ir], u = Zy[yu * QW + ir];
            const T dl = Zd[yd * QW + xl], dr = Zd[yd * QW + xr], ul = Zd[yu * QW + xl], ur = Zd[yu * QW + xr];
            T* w = Zc + jr * QW + ir;
            if (inner) {
                *w = (Bc[jr * QW + ir] - (c.fc * (dl + dr + ul + ur) + c.fey * (d + u) + c.fex * (l + r))) *
                     c.invd[1][1];
            } else {
                const int i = zx + ii, j = zy + jj;
                if (unsigned(i) >= unsigned(M) || unsigned(j) >= unsigned(N)) continue;
                *w = (Bc[jr * QW + ir] - fem_off_vals(c, i, j, dl, d, dr, l, r, ul, u, ur)) *
                     pick3(c.invd, cls(i, M), cls(j, N));
            }
        }
        __syncthreads();
    }
    auto zat = [&](int ii, int jj) -> T { return Z[qidx(ii, jj)]; };
    auto resid = [&](int ii, int jj) -> T {
        const int i = zx + ii, j = zy + jj;
        T off = fem_off_vals(c, i, j, zat(ii - 1, jj - 1), zat(ii, jj - 1), zat(ii + 1, jj - 1), zat(ii - 1, jj),
                             zat(ii + 1, jj), zat(ii - 1, jj + 1), zat(ii, jj + 1), zat(ii + 1, jj + 1));
        return B[qidx(ii, jj)] - pick3(c.d, cls(i, M), cls(j, N)) * zat(ii, jj) - off;
    };
    for (int jj = ZH + warp; jj < ZH + TY; jj += NW) {
        const int j = zy + jj;
        if (j >= N) break;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int ii = ZH + lane + 32 * h;
            const int i = zx + ii;
            if (ii < ZH + TX && i < M) a.zout[i + M * j] = zat(ii, jj);
        }
    }
    // The residual passes give a warp 32 points of one column parity, so
    // each of the residual's reads is 32 consecutive words of one quarter
    // (consecutive window columns alternate quarters: a warp over them
    // would read two quarters' words in the same banks).
    static_assert(ZH % 2 == 0 && (RW + 1) / 2 <= 32 && TX / 2 <= 32, "one warp per colour row");
    if (MODE == 0) {
        // residuals on the interior and one ring, held as four colour
        // quarters (ring column/row ZH-1+2k and ZH+2k share index k), then
        // P^T onto coarse nodes
        constexpr int RQ = (RW + 1) / 2, RQN = RQ * ((RH + 1) / 2);
        static_assert(4 * RQN <= RW * RH, "ring quarters fit the ring array");
        auto ridx = [](int ii, int jj) {
            return ((ii & 1) + 2 * (jj & 1)) * RQN + ((jj - (ZH - 1)) >> 1) * RQ + ((ii - (ZH - 1)) >> 1);
        };
        for (int jr = warp; jr < RH; jr += NW) {
            const int jj = ZH - 1 + jr, j = zy + jj;
#pragma unroll
            for (int ci = 0; ci < 2; ci++) {
                const int ii = ZH - 1 + (1 - ci) + 2 * lane;   // ZH - 1 is odd
                if (ii >= ZH - 1 + RW) continue;
                const int i = zx + ii;
                R[ridx(ii, jj)] = (unsigned(i) < unsigned(M) && unsigned(j) < unsigned(N)) ? resid(ii, jj) : T(0);
            }
        }
        __syncthreads();
        const int Mc = (M - 1) / 2 + 1, Nc = (N - 1) / 2 + 1;
        constexpr int CX = TX / 2, CY = TY / 2;
        for (int t = threadIdx.x; t < CX * CY; t += G::NT) {
            const int q = t / CX;
            const int I = x0 / 2 + (t - q * CX), J = y0 / 2 + q;
            if (I >= Mc || J >= Nc) continue;
            a.bc[I + Mc * J] = TC(fem_restrict_by<T>(M, N, [&](int i, int j) { return R[ridx(i - zx, j - zy)]; }, I, J));
        }
    } else if (a.norm) {
        double s = 0;
        for (int jj = ZH + warp; jj < ZH + TY; jj += NW) {
            const int j = zy + jj;
            if (j >= N) break;
#pragma unroll
            for (int ci = 0; ci < 2; ci++) {
                const int ii = ZH + ci + 2 * lane;
                if (ii < ZH + TX && zx + ii < M) {
                    double r = double(resid(ii, jj));
                    s += r * r;
                }
            }
        }
        s = block_sum(s);
        double total;
        if (grid_sum(s, a.rd, &total) && threadIdx.x == 0) solve_decide(a.ctl, total, 1, a.use_cond, a.h);
    }
}

// ------------------------------------- register-blocked node-centred tile
// The FEM counterpart of cc_rtile: the same window computation as fem_tile
// (64 x 64 nodes, even origin, eight four-colour phases on a shrinking
// region, the same update, residual and restriction arithmetic), with thread
// (warp w, lane t) holding columns 2t, 2t+1 and rows 8w..8w+7 in registers.
// A colour (ci, cj) is column ci of the thread's pair on the rows of parity
// cj; the eight neighbours are the thread's own registers, the facing
// column of the adjacent lane (shuffles) and, across warps, the first and
// last rows through a small shared array.
template <typename T>
struct FEMReg {
    static constexpr int R = 8;
    static constexpr int NWARP = 8;
    static constexpr int NT = 32 * NWARP;
    static constexpr int CW = 64, CH = R * NWARP;
    static constexpr int K = 8;                 // two four-colour sweeps
    static constexpr int ZH = 10;               // K + 1 rings, rounded up to even
    static constexpr int TX = CW - 2 * ZH, TY = CH - 2 * ZH;
};

template <typename T, int MODE, typename TC = T, int MINB = 2>
__global__ void __launch_bounds__(FEMReg<T>::NT, MINB) fem_rtile(FEMc<T> c, TileArgs<T, TC> a) {
    using G = FEMReg<T>;
    constexpr int R = G::R, CW = G::CW, CH = G::CH, K = G::K, ZH = G::ZH, NWARP = G::NWARP;
    __shared__ __align__(16) T edge[2][2][NWARP][CW];
    const int M = c.M, N = c.N;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int zx = blockIdx.x * G::TX - ZH, zy = blockIdx.y * G::TY - ZH;
    const int i0 = zx + 2 * lane, j0 = zy + warp * R;
    const bool read_z = MODE == 1 || !a.zero_init;
    T z[R][2], b[R][2];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int j = j0 + r;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int i = i0 + h;
            const bool in = unsigned(j) < unsigned(N) && unsigned(i) < unsigned(M);
            b[r][h] = in ? a.b[i + long(M) * j] : T(0);
            z[r][h] = (in && read_z) ? a.zin[i + long(M) * j] : T(0);
        }
    }
    if constexpr (MODE == 1) {
        // prolongation: coarse node (I, J) sits on fine node (2I, 2J); the
        // thread's fine rows j0..j0+7 use coarse rows J0..J0+4 of columns I
        // (its own) and I+1 (the next lane's)
        const int Mc = (M - 1) / 2 + 1, Nc = (N - 1) / 2 + 1, I = i0 >> 1, J0 = j0 >> 1;
        constexpr int CR = R / 2 + 1;
        T cc[CR], cp[CR];
#pragma unroll
        for (int q = 0; q < CR; q++) {
            const int J = J0 + q;
            const bool rin = unsigned(J) < unsigned(Nc);
            cc[q] = (rin && unsigned(I) < unsigned(Mc)) ? T(a.zc[I + long(Mc) * J]) : T(0);
            cp[q] = shfl_dn1(cc[q]);
            if (lane == 31) cp[q] = (rin && unsigned(I + 1) < unsigned(Mc)) ? T(a.zc[I + 1 + long(Mc) * J]) : T(0);
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int j = j0 + r, q = r >> 1;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int i = i0 + h;
                if (!(unsigned(i) < unsigned(M) && unsigned(j) < unsigned(N)) || j == 0) continue;
                const T c00 = cc[q];
                T v;
                if (h == 0 && (r & 1) == 0) v = c00;
                else if (h == 1 && (r & 1) == 0) v = T(0.5) * (c00 + cp[q]);
                else if (h == 0) v = T(0.5) * (c00 + cc[q + 1]);
                else v = T(0.25) * (c00 + cp[q] + cc[q + 1] + cp[q + 1]);
                z[r][h] += v;
            }
        }
    }
#pragma unroll
    for (int ph = 0; ph < K; ph++) {
        const int colour = MODE == 1 ? 3 - (ph & 3) : (ph & 3);
        const int ci = colour & 1, cj = colour >> 1, oc = 1 - ci;
        T(*eb)[NWARP][CW] = edge[ph & 1];
        reinterpret_cast<typename std::conditional<sizeof(T) == 8, double2, float2>::type*>(&eb[0][warp][0])[lane] =
            {z[0][0], z[0][1]};
        reinterpret_cast<typename std::conditional<sizeof(T) == 8, double2, float2>::type*>(&eb[1][warp][0])[lane] =
            {z[R - 1][0], z[R - 1][1]};
        __syncthreads();
        T below[2], above[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            below[h] = warp > 0 ? eb[1][warp - 1][2 * lane + h] : T(0);
            above[h] = warp < NWARP - 1 ? eb[0][warp + 1][2 * lane + h] : T(0);
        }
        // the other column of the thread (rows -1..R) and the facing column
        // of the adjacent lane: left of column 0, right of column 1
        T own[R + 2], nb[R + 2];
#pragma unroll
        for (int k = 0; k < R + 2; k++) {
            own[k] = k == 0 ? below[oc] : (k == R + 1 ? above[oc] : z[k == 0 || k == R + 1 ? 0 : k - 1][oc]);
            nb[k] = ci == 0 ? shfl_up1(own[k]) : shfl_dn1(own[k]);
        }
#pragma unroll
        for (int r = 0; r < R; r++) {
            if ((r & 1) != cj) continue;
            const int i = i0 + ci, j = j0 + r;
            const int ii = 2 * lane + ci, jj = warp * R + r;
            const T d = r > 0 ? z[r > 0 ? r - 1 : 0][ci] : below[ci];
            const T u = r < R - 1 ? z[r < R - 1 ? r + 1 : R - 1][ci] : above[ci];
            // rows r-1, r, r+1 sit at k = r, r+1, r+2 of own[] and nb[]
            const T l = ci == 0 ? nb[r + 1] : own[r + 1];
            const T rr = ci == 0 ? own[r + 1] : nb[r + 1];
            const T dl = ci == 0 ? nb[r] : own[r];
            const T dr = ci == 0 ? own[r] : nb[r];
            const T ul = ci == 0 ? nb[r + 2] : own[r + 2];
            const T ur = ci == 0 ? own[r + 2] : nb[r + 2];
            const bool upd = ii >= ph + 1 && ii <= CW - 2 - ph && jj >= ph + 1 && jj <= CH - 2 - ph &&
                             unsigned(i) < unsigned(M) && unsigned(j) < unsigned(N);
            const T zn = (b[r][ci] - fem_off_vals(c, i, j, dl, d, dr, l, rr, ul, u, ur)) *
                         pick3(c.invd, cls(i, M), cls(j, N));
            z[r][ci] = upd ? zn : z[r][ci];
        }
    }
    const bool lanein = 2 * lane >= ZH && 2 * lane < ZH + G::TX;
#pragma unroll
    for (int r = 0; r < R; r++) {
        const int jj = warp * R + r, j = j0 + r;
        if (!lanein || jj < ZH || jj >= ZH + G::TY || j >= N) continue;
#pragma unroll
        for (int h = 0; h < 2; h++)
            if (i0 + h < M) a.zout[i0 + h + long(M) * j] = z[r][h];
    }
    const bool want_resid = MODE == 0 ? a.bc != nullptr : a.norm != 0;
    if (!want_resid) return;
    // the final iterate's first and last rows across warps once more
    {
        T(*eb)[NWARP][CW] = edge[K & 1];
        eb[0][warp][2 * lane] = z[0][0];
        eb[0][warp][2 * lane + 1] = z[0][1];
        eb[1][warp][2 * lane] = z[R - 1][0];
        eb[1][warp][2 * lane + 1] = z[R - 1][1];
    }
    __syncthreads();
    T below[2], above[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        below[h] = warp > 0 ? edge[K & 1][1][warp - 1][2 * lane + h] : T(0);
        above[h] = warp < NWARP - 1 ? edge[K & 1][0][warp + 1][2 * lane + h] : T(0);
    }
    // residual of row r at both columns
    auto zrow = [&](int k, int h) -> T { return k < 0 ? below[h] : (k >= R ? above[h] : z[k < 0 ? 0 : (k >= R ? R - 1 : k)][h]); };
    auto resid_row = [&](int r, T& r0, T& r1) {
        const int j = j0 + r;
        const T up1 = shfl_up1(zrow(r, 1)), up1d = shfl_up1(zrow(r - 1, 1)), up1u = shfl_up1(zrow(r + 1, 1));
        const T dn0 = shfl_dn1(zrow(r, 0)), dn0d = shfl_dn1(zrow(r - 1, 0)), dn0u = shfl_dn1(zrow(r + 1, 0));
        {
            const int i = i0;
            const T off = fem_off_vals(c, i, j, up1d, zrow(r - 1, 0), zrow(r - 1, 1), up1, zrow(r, 1), up1u,
                                       zrow(r + 1, 0), zrow(r + 1, 1));
            r0 = b[r][0] - pick3(c.d, cls(i, M), cls(j, N)) * z[r][0] - off;
        }
        {
            const int i = i0 + 1;
            const T off = fem_off_vals(c, i, j, zrow(r - 1, 0), zrow(r - 1, 1), dn0d, zrow(r, 0), dn0,
                                       zrow(r + 1, 0), zrow(r + 1, 1), dn0u);
            r1 = b[r][1] - pick3(c.d, cls(i, M), cls(j, N)) * z[r][1] - off;
        }
        const bool rowin = unsigned(j) < unsigned(N);
        if (!(rowin && unsigned(i0) < unsigned(M))) r0 = T(0);
        if (!(rowin && unsigned(i0 + 1) < unsigned(M))) r1 = T(0);
    };
    if constexpr (MODE == 0) {
        // P^T: coarse node (I, J) on fine (2I, 2J) gathers rows 2J-1..2J+1
        // and columns 2I-1..2I+1 (half weights off the centre line); the row
        // below the strip comes from the warp below, the column left of the
        // thread's pair from the adjacent lane
        __shared__ T rlast[NWARP][CW];
        T rl0, rl1;
        resid_row(R - 1, rl0, rl1);
        rlast[warp][2 * lane] = rl0;
        rlast[warp][2 * lane + 1] = rl1;
        __syncthreads();
        T pr0 = warp > 0 ? rlast[warp - 1][2 * lane] : T(0);
        T pr1 = warp > 0 ? rlast[warp - 1][2 * lane + 1] : T(0);
        const int Mc = (M - 1) / 2 + 1, Nc = (N - 1) / 2 + 1, I = i0 >> 1;
#pragma unroll
        for (int k = 0; k < R / 2; k++) {
            T c0, c1, n0, n1;
            resid_row(2 * k, c0, c1);
            if (2 * k + 1 == R - 1) {
                n0 = rl0;
                n1 = rl1;
            } else {
                resid_row(2 * k + 1, n0, n1);
            }
            // column 2I-1: the previous lane's second column
            const T pl = shfl_up1(pr1), cl = shfl_up1(c1), nl = shfl_up1(n1);
            const int jj = warp * R + 2 * k, J = (j0 >> 1) + k;
            const bool ok = lanein && jj >= ZH && jj < ZH + G::TY && unsigned(I) < unsigned(Mc) &&
                            unsigned(J) < unsigned(Nc);
            if (ok) {
                T sum = 0;
                if (J > 0) {
                    const T rows[3][3] = {{pl, pr0, pr1}, {cl, c0, c1}, {nl, n0, n1}};
#pragma unroll
                    for (int dj = -1; dj <= 1; dj++) {
                        const int jf = 2 * J + dj;
                        if (jf < 0 || jf >= N) continue;
                        const T wy = dj == 0 ? T(1) : T(0.5);
#pragma unroll
                        for (int di = -1; di <= 1; di++) {
                            const int ifn = 2 * I + di;
                            if (ifn < 0 || ifn >= M) continue;
                            const T wx = di == 0 ? T(1) : T(0.5);
                            sum += wx * wy * rows[dj + 1][di + 1];
                        }
                    }
                }
                a.bc[I + long(Mc) * J] = TC(sum);
            }
            pr0 = n0;
            pr1 = n1;
        }
    } else {
        double s = 0;
#pragma unroll
        for (int r = 0; r < R; r++) {
            T r0, r1;
            resid_row(r, r0, r1);
            const int jj = warp * R + r, j = j0 + r;
            if (!lanein || jj < ZH || jj >= ZH + G::TY || j >= N) continue;
            if (i0 < M) s += double(r0) * double(r0);
            if (i0 + 1 < M) s += double(r1) * double(r1);
        }
        s = block_sum(s);
        double total;
        if (grid_sum(s, a.rd, &total) && threadIdx.x == 0) solve_decide(a.ctl, total, 1, a.use_cond, a.h);
    }
}

// ---------------------------------------------------- CTA-resident levels
template <typename T>
struct CCStack {
    int nl;
    CCc<T> lv[MAXLEV];
    int off[MAXLEV];     // element offsets of z_l; b_l follows z_l
    int nu1, nu2, ncoarse;
    const T* dinv;       // inverse of the last level's operator (solved exactly), or null
};

template <typename T>
struct FEMStack {
    int nl;
    FEMc<T> lv[MAXLEV];
    int off[MAXLEV];     // z_l, then b_l, then r_l
    int nu1, nu2, ncoarse;
    const T* dinv;       // inverse of the last level's operator (solved exactly), or null
};

/** z = inv b for the CTA's last level (N unknowns, inv row-major in global
 * memory): warp w takes rows w, w + 32, ...; lanes split each row. */
template <typename T>
__device__ void cta_direct(const T* __restrict__ inv, int N, const T* b, T* z) {
    const int lane = threadIdx.x & 31;
    for (int r = threadIdx.x >> 5; r < N; r += blockDim.x >> 5) {
        T s = 0;
        for (int k = lane; k < N; k += 32) s += inv[size_t(r) * N + k] * b[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) z[r] = s;
    }
    __syncthreads();
}

/** z = X b for a dense row-major N x N inverse X with row pitch P (a
 * multiple of 4, the pad zero), one warp per row: 16-byte loads, four
 * independent partial sums per lane, so a warp keeps 2-4 KB of its row in
 * flight. b is staged in shared memory (zero-padded to P). The exact solve
 * of a coarse level over the whole GPU. */
template <typename T>
__global__ void __launch_bounds__(256) direct_matvec_k(const T* __restrict__ X, int N, int P,
                                                       const T* __restrict__ b, T* __restrict__ z) {
    using V = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
    constexpr int E = int(sizeof(V) / sizeof(T));   // elements per vector
    extern __shared__ __align__(16) unsigned char dm_raw[];
    T* sb = reinterpret_cast<T*>(dm_raw);
    for (int k = threadIdx.x; k < P; k += blockDim.x) sb[k] = k < N ? b[k] : T(0);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (r >= N) return;
    const V* row = reinterpret_cast<const V*>(X + size_t(r) * P);
    const V* bv = reinterpret_cast<const V*>(sb);
    const int nv = P / E;
    T acc[4] = {0, 0, 0, 0};
    int q = lane;
    for (; q + 96 < nv; q += 128) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const V x = __ldg(row + q + 32 * u), y = bv[q + 32 * u];
            if constexpr (E == 2) acc[u] += x.x * y.x + x.y * y.y;
            else acc[u] += x.x * y.x + x.y * y.y + x.z * y.z + x.w * y.w;
        }
    }
    for (; q < nv; q += 32) {
        const V x = __ldg(row + q), y = bv[q];
        if constexpr (E == 2) acc[0] += x.x * y.x + x.y * y.y;
        else acc[0] += x.x * y.x + x.y * y.y + x.z * y.z + x.w * y.w;
    }
    T s = (acc[0] + acc[1]) + (acc[2] + acc[3]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) z[r] = s;
}

/** Copies a dense N x N matrix into rows of pitch P >= N (zero pad), in
 * FP64 and FP32. */
__global__ void pad_rows_k(const double* __restrict__ A, int N, int P, double* __restrict__ X64,
                           float* __restrict__ X32) {
    const long tot = long(N) * P;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < tot; k += long(gridDim.x) * blockDim.x) {
        const long r = k / P, c = k - r * P;
        const double v = c < N ? A[r * N + c] : 0.;
        X64[k] = v;
        X32[k] = float(v);
    }
}

/** Gauss-Jordan inversion on the device, in place and without pivoting (the
 * coarse FEM operators are symmetric positive definite once their Dirichlet
 * rows, which hold only a diagonal, are eliminated first; those come first
 * in the row order). A is assembled from nine stencil planes. */
__global__ void gj_assemble_k(const double* __restrict__ S, int m, int n, double* __restrict__ A) {
    const int N = m * n;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    const int j = k / m, i = k - j * m;
    for (int d = 0; d < 9; d++) {
        const int ii = i + d % 3 - 1, jj = j + d / 3 - 1;
        if (ii < 0 || ii >= m || jj < 0 || jj >= n) continue;
        A[size_t(k) * N + ii + size_t(m) * jj] += S[size_t(d) * N + k];
    }
}
/** Step k: the scaled pivot row rk and the pivot column ck (old values). */
__global__ void gj_pivot_k(const double* __restrict__ A, int N, int k, double* __restrict__ rk,
                           double* __restrict__ ck, int* bad) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= N) return;
    const double p = A[size_t(k) * N + k];
    if (q == 0 && !(fabs(p) > 1e-300 && isfinite(p))) atomicOr(bad, 1);
    rk[q] = (q == k ? 1. : A[size_t(k) * N + q]) / p;
    ck[q] = q == k ? 0. : A[size_t(q) * N + k];
}
__global__ void gj_update_k(double* __restrict__ A, int N, int k, const double* __restrict__ rk,
                            const double* __restrict__ ck) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (q >= N) return;
    double* a = A + size_t(i) * N + q;
    if (i == k) *a = rk[q];
    else *a = (q == k ? 0. : *a) - ck[i] * rk[q];
}

/** Row loops of the CTA-resident levels: warp w takes rows w, w+nw, ...;
 * lanes take columns, so no index division is needed. */
#define CTA_ROWS(j, j0, jstep, nrows) \
    for (int j = (j0) + (threadIdx.x >> 5) * (jstep); j < (nrows); j += (blockDim.x >> 5) * (jstep))

/** One colour of a whole-level sweep inside the CTA. */
template <typename T>
__device__ void cta_sweep(const CCc<T>& c, T* z, const T* b, int color) {
    const int lane = threadIdx.x & 31;
    CTA_ROWS(j, 0, 1, c.n) {
        for (int i = 2 * lane + ((color ^ j) & 1); i < c.m; i += 64) {
            T* w = z + i + c.m * j;
            *w = op_relaxed(c, w, b[i + c.m * j], c.m, i, j);
        }
    }
    __syncthreads();
}

template <typename T>
__device__ void cta_sweep(const FEMc<T>& c, T* z, const T* b, int color) {
    const int ci = color & 1, cj = color >> 1, lane = threadIdx.x & 31;
    CTA_ROWS(j, cj, 2, c.N) {
        for (int i = ci + 2 * lane; i < c.M; i += 64) {
            T* w = z + i + c.M * j;
            *w = op_relaxed(c, w, b[i + c.M * j], c.M, i, j);
        }
    }
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(CTA_THREADS) cc_cta_cycle(CCStack<T> st, const T* __restrict__ gb,
                                                           T* __restrict__ gz, int zero_init) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    const int lane = threadIdx.x & 31;
    {
        const CCc<T>& c0 = st.lv[0];
        T* z = sm + st.off[0];
        T* b = z + c0.m * c0.n;
        const int tot = c0.m * c0.n;
        for (int k = threadIdx.x; k < tot; k += blockDim.x) {
            b[k] = gb[k];
            z[k] = zero_init ? T(0) : gz[k];
        }
        for (int l = 1; l < st.nl; l++) {
            T* zl = sm + st.off[l];
            for (int k = threadIdx.x; k < st.lv[l].m * st.lv[l].n; k += blockDim.x) zl[k] = T(0);
        }
    }
    __syncthreads();
    for (int l = 0; l < st.nl - 1; l++) {
        const CCc<T>& c = st.lv[l];
        T* z = sm + st.off[l];
        T* b = z + c.m * c.n;
        for (int s = 0; s < st.nu1; s++) {
            cta_sweep(c, z, b, 0);
            cta_sweep(c, z, b, 1);
        }
        const CCc<T>& cc = st.lv[l + 1];
        T* bcn = sm + st.off[l + 1] + cc.m * cc.n;
        CTA_ROWS(J, 0, 1, cc.n) {
            for (int I = lane; I < cc.m; I += 32) {
                T s = 0;
                for (int dj = 0; dj < 2; dj++)
                    for (int di = 0; di < 2; di++) {
                        int i = 2 * I + di, j = 2 * J + dj;
                        s += op_resid(c, z + i + c.m * j, b[i + c.m * j], c.m, i, j);
                    }
                bcn[I + cc.m * J] = T(0.25) * s;
            }
        }
        __syncthreads();
    }
    {
        const CCc<T>& c = st.lv[st.nl - 1];
        T* z = sm + st.off[st.nl - 1];
        T* b = z + c.m * c.n;
        if (st.dinv) {
            cta_direct(st.dinv, c.m * c.n, b, z);
        } else {
            int ns = st.nl > 1 ? st.ncoarse : st.nu1 + st.nu2;
            for (int s = 0; s < ns; s++) {
                cta_sweep(c, z, b, 0);
                cta_sweep(c, z, b, 1);
            }
        }
    }
    for (int l = st.nl - 2; l >= 0; l--) {
        const CCc<T>& c = st.lv[l];
        T* z = sm + st.off[l];
        T* b = z + c.m * c.n;
        const T* zc = sm + st.off[l + 1];
        CTA_ROWS(j, 0, 1, c.n) {
            for (int i = lane; i < c.m; i += 32) z[i + c.m * j] += cc_interp(c, zc, i, j);
        }
        __syncthreads();
        for (int s = 0; s < st.nu2; s++) {
            cta_sweep(c, z, b, 1);
            cta_sweep(c, z, b, 0);
        }
    }
    {
        const CCc<T>& c0 = st.lv[0];
        const T* z = sm + st.off[0];
        for (int k = threadIdx.x; k < c0.m * c0.n; k += blockDim.x) gz[k] = z[k];
    }
}

template <typename T>
__global__ void __launch_bounds__(CTA_THREADS) fem_cta_cycle(FEMStack<T> st, const T* __restrict__ gb,
                                                            T* __restrict__ gz, int zero_init) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    const int lane = threadIdx.x & 31;
    {
        const FEMc<T>& c0 = st.lv[0];
        T* z = sm + st.off[0];
        T* b = z + c0.M * c0.N;
        for (int k = threadIdx.x; k < c0.M * c0.N; k += blockDim.x) {
            b[k] = gb[k];
            z[k] = zero_init ? T(0) : gz[k];
        }
        for (int l = 1; l < st.nl; l++) {
            T* zl = sm + st.off[l];
            for (int k = threadIdx.x; k < st.lv[l].M * st.lv[l].N; k += blockDim.x) zl[k] = T(0);
        }
    }
    __syncthreads();
    for (int l = 0; l < st.nl - 1; l++) {
        const FEMc<T>& c = st.lv[l];
        const int tot = c.M * c.N;
        T* z = sm + st.off[l];
        T* b = z + tot;
        T* r = b + tot;
        for (int s = 0; s < st.nu1; s++)
            for (int q = 0; q < 4; q++) cta_sweep(c, z, b, q);
        CTA_ROWS(j, 0, 1, c.N) {
            for (int i = lane; i < c.M; i += 32) {
                int k = i + c.M * j;
                r[k] = op_resid(c, z + k, b[k], c.M, i, j);
            }
        }
        __syncthreads();
        const FEMc<T>& cc = st.lv[l + 1];
        T* bcn = sm + st.off[l + 1] + cc.M * cc.N;
        CTA_ROWS(J, 0, 1, cc.N) {
            for (int I = lane; I < cc.M; I += 32) bcn[I + cc.M * J] = fem_restrict_at(c.M, c.N, r, c.M, 0, 0, I, J);
        }
        __syncthreads();
    }
    {
        const FEMc<T>& c = st.lv[st.nl - 1];
        T* z = sm + st.off[st.nl - 1];
        T* b = z + c.M * c.N;
        if (st.dinv) {
            cta_direct(st.dinv, c.M * c.N, b, z);
        } else {
            int ns = st.nl > 1 ? st.ncoarse : st.nu1 + st.nu2;
            for (int s = 0; s < ns; s++)
                for (int q = 0; q < 4; q++) cta_sweep(c, z, b, q);
        }
    }
    for (int l = st.nl - 2; l >= 0; l--) {
        const FEMc<T>& c = st.lv[l];
        const int tot = c.M * c.N;
        T* z = sm + st.off[l];
        T* b = z + tot;
        const T* zc = sm + st.off[l + 1];
        CTA_ROWS(j, 0, 1, c.N) {
            for (int i = lane; i < c.M; i += 32) z[i + c.M * j] += fem_interp(c, zc, i, j);
        }
        __syncthreads();
        for (int s = 0; s < st.nu2; s++)
            for (int q = 3; q >= 0; q--) cta_sweep(c, z, b, q);
    }
    {
        const FEMc<T>& c0 = st.lv[0];
        const T* z = sm + st.off[0];
        for (int k = threadIdx.x; k < c0.M * c0.N; k += blockDim.x) gz[k] = z[k];
    }
}

// ------------------------------------------------------- whole-grid kernels
template <class OP>
__device__ __forceinline__ void grid_ij(const OP& c, long k, int& i, int& j) {
    j = int(k / op_m(c));
    i = int(k - long(j) * op_m(c));
}

/** Rows of one warp's strip in strip_walk. */
static constexpr int STRIP_ROWS = 16;

/** Walk over an m x n grid by strips of 32 columns and STRIP_ROWS rows, one
 * warp per strip (warps take strips a grid's warps apart): lane t calls
 * f(k, i, j) for column i = strip column + t down the strip's rows. The
 * stencil's neighbours in rows j-1 and j+1 are the rows the same warp has
 * just read or reads next, so they come from L1: z and b cross DRAM once. */
template <class F>
__device__ __forceinline__ void strip_walk(int m, int n, F f) {
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const int sx = (m + 31) >> 5, sy = (n + STRIP_ROWS - 1) / STRIP_ROWS, ns = sx * sy;
    for (int sidx = blockIdx.x * wpb + (threadIdx.x >> 5); sidx < ns; sidx += gridDim.x * wpb) {
        const int sj = sidx / sx, i = (sidx - sj * sx) * 32 + lane;
        if (i >= m) continue;
        const int j0 = sj * STRIP_ROWS, j1 = min(j0 + STRIP_ROWS, n);
#pragma unroll 4
        for (int j = j0; j < j1; j++) f(long(j) * m + i, i, j);
    }
}

/** ||b - A z||^2 accumulated in FP64, then the solve decision. */
template <typename T, class OP>
__global__ void resid_norm_k(OP c, const T* __restrict__ z, const T* __restrict__ b, Reduce rd, SolveCtl* ctl,
                             int count_cycle, int use_cond, cudaGraphConditionalHandle h) {
    double s = 0;
    strip_walk(op_m(c), op_n(c), [&](long k, int i, int j) {
        double r = double(op_resid(c, z + k, b[k], op_m(c), i, j));
        s += r * r;
    });
    s = block_sum(s);
    double total;
    if (grid_sum(s, rd, &total) && threadIdx.x == 0) solve_decide(ctl, total, count_cycle, use_cond, h);
}

/** The start of a solve in one pass: ||b||^2 and ||b - A z0||^2, then the
 * first decision. A zero source is done at once with z = 0 (the shim and
 * this library agree on that convention): the last block, which every other
 * block has finished reading z before, zeroes it. With r32 (mixed
 * precision) the residual is also written in FP32, the source of the first
 * FP32 V-cycle. */
template <typename T, class OP>
__global__ void first_check_k(OP c, T* __restrict__ z, const T* __restrict__ b, Reduce rd, SolveCtl* ctl,
                              int use_cond, cudaGraphConditionalHandle h, float* __restrict__ r32 = nullptr) {
    __shared__ int zero_src;
    double sb = 0, sr = 0;
    const long tot = long(op_m(c)) * op_n(c);
    strip_walk(op_m(c), op_n(c), [&](long k, int i, int j) {
        double bv = double(b[k]);
        double r = double(op_resid(c, z + k, b[k], op_m(c), i, j));
        if (r32) r32[k] = float(r);
        sb += bv * bv;
        sr += r * r;
    });
    sb = block_sum(sb);
    __syncthreads();
    sr = block_sum(sr);
    double b2, r2;
    if (!grid_sum2(sb, sr, rd, &b2, &r2)) return;
    if (threadIdx.x == 0) {
        ctl->bnorm2 = b2;
        ctl->it = 0;
        ctl->done = 0;
        ctl->status = 0;
        solve_decide(ctl, b2 == 0. ? 0. : r2, 0, use_cond, h);
        zero_src = b2 == 0.;
    }
    __syncthreads();
    if (zero_src)
        for (long k = threadIdx.x; k < tot; k += blockDim.x) z[k] = T(0);
}

/** FP64 residual of an FP64 iterate written as FP32 (a refinement step),
 * with its FP64 norm and the solve decision. */
template <class OP>
__global__ void resid_to32_k(OP c, const double* __restrict__ z, const double* __restrict__ b,
                             float* __restrict__ r32, Reduce rd, SolveCtl* ctl, int count_cycle, int use_cond,
                             cudaGraphConditionalHandle h) {
    double s = 0;
    strip_walk(op_m(c), op_n(c), [&](long k, int i, int j) {
        double r = op_resid(c, z + k, b[k], op_m(c), i, j);
        r32[k] = float(r);
        s += r * r;
    });
    s = block_sum(s);
    double total;
    if (grid_sum(s, rd, &total) && threadIdx.x == 0) solve_decide(ctl, total, count_cycle, use_cond, h);
}

template <typename T, class OP>
__global__ void apply_k(OP c, const T* __restrict__ z, T* __restrict__ y) {
    const long tot = long(op_m(c)) * op_n(c);
    long k = blockIdx.x * long(blockDim.x) + threadIdx.x;
    if (k >= tot) return;
    int i, j;
    grid_ij(c, k, i, j);
    y[k] = pick3(c.d, cls(i, op_m(c)), cls(j, op_n(c))) * z[k] + op_off(c, z + k, op_m(c), i, j);
}

template <typename T, class OP>
__global__ void resid_out_k(OP c, const T* __restrict__ z, const T* __restrict__ b, T* __restrict__ r, Reduce rd,
                            double* out) {
    double s = 0;
    strip_walk(op_m(c), op_n(c), [&](long k, int i, int j) {
        T v = op_resid(c, z + k, b[k], op_m(c), i, j);
        if (r) r[k] = v;
        s += double(v) * double(v);
    });
    s = block_sum(s);
    double total;
    if (grid_sum(s, rd, &total) && threadIdx.x == 0) *out = sqrt(total);
}

__global__ void add_f32_to_f64(double* __restrict__ z, const float* __restrict__ e, long n) {
    long k = blockIdx.x * long(blockDim.x) + threadIdx.x;
    if (k < n) z[k] += double(e[k]);
}

/** The same addition four points a thread, with 16-byte loads and stores
 * (z and e 16-byte aligned); the last n % 4 points one by one. */
__global__ void add_f32_to_f64_x4(double* __restrict__ z, const float* __restrict__ e, long n) {
    const long q = blockIdx.x * long(blockDim.x) + threadIdx.x, k = 4 * q;
    if (k + 3 < n) {
        const float4 ev = reinterpret_cast<const float4*>(e)[q];
        double2* z2 = reinterpret_cast<double2*>(z) + 2 * q;
        double2 a = z2[0], c = z2[1];
        a.x += double(ev.x);
        a.y += double(ev.y);
        c.x += double(ev.z);
        c.y += double(ev.w);
        z2[0] = a;
        z2[1] = c;
    } else {
        for (long t = k; t < n; t++) z[t] += double(e[t]);
    }
}

// =================================================================== host
static inline int nblk(long n, int t = 256) { return int((n + t - 1) / t); }
/** Blocks of 256 threads that the current GPU holds at once: 6 per SM for
 * the reduction kernels' 40 registers per thread. */
static inline int resident_blocks() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        sms = 148;
    return 6 * std::max(1, sms);
}
/** Blocks of a whole-grid reduction over n points: one resident wave at
 * most, so the partial sums stay few and the last block's sum short. */
static inline int rblocks(long n) { return std::max(1, std::min({MAX_PARTIALS, nblk(n, 256), resident_blocks()})); }
/** Blocks of 256 threads for a strip_walk over an m x n grid: one warp per
 * strip, one resident wave at most, few enough for grid_sum2's partials. */
static inline int sblocks(int m, int n) {
    const long strips = long((m + 31) / 32) * ((n + STRIP_ROWS - 1) / STRIP_ROWS);
    return int(std::max(1L, std::min({long(MAX_PARTIALS / 2), (strips + 7) / 8, long(resident_blocks())})));
}

/** Per-level description in double precision, converted per precision. */
struct LevelD {
    int m, n;              // cell-centred: cells; FEM: nodes (M, N)
    double ox, oy;         // cell-centred couplings
    double d[3][3];
    signed char gL, gR, gD, gU;
};

/** Which tile kernels the V-cycles launch, read once: the shared-memory
 * ones (0, default), the register-blocked ones with two CTAs per SM
 * (1, VDI_MG_TILE=reg) or one CTA per SM and its whole register file
 * (2, VDI_MG_TILE=reg1), or for FP64 cell-centred levels the persistent
 * TMA-fed register tile (3, VDI_MG_TILE=tma; other levels as in 0). */
static int reg_tile_mode() {
    static int v = -1;
    if (v < 0) {
        const char* e = getenv("VDI_MG_TILE");
        v = !e ? 0
               : (std::strcmp(e, "reg") == 0 ? 1
                  : (std::strcmp(e, "reg1") == 0 ? 2 : (std::strcmp(e, "tma") == 0 ? 3 : 0)));
    }
    return v;
}
static bool use_reg_tile() { const int v = reg_tile_mode(); return v == 1 || v == 2; }

/** Launches of the persistent tile issued so far (a captured graph's count
 * once, at capture). */
static std::atomic<long long> g_ptile_launches{0};

int mg_tile_path(long long* persistent_launches) {
    if (persistent_launches) *persistent_launches = g_ptile_launches.load(std::memory_order_relaxed);
    return reg_tile_mode();
}

/** The driver's tensor-map encoder, looked up once through the runtime so
 * the library does not link libcuda itself; null when unavailable. */
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        else
            cudaGetLastError();
    }
    return encode;
}

/** A 2D tensor map of an m x n FP64 array (row pitch m) with 64 x 64 boxes,
 * zero fill outside the array: one per array, cached. False when the array
 * cannot be described (odd m, unaligned base). */
static bool tile_tensor_map(const double* p, int m, int n, CUtensorMap* out) {
    if ((m & 1) || (reinterpret_cast<uintptr_t>(p) & 15)) return false;
    struct Entry {
        const double* p;
        int m, n;
        CUtensorMap map;
    };
    static std::mutex mu;
    static std::vector<Entry> cache;
    std::lock_guard<std::mutex> lock(mu);
    for (auto& e : cache)
        if (e.p == p && e.m == m && e.n == n) {
            *out = e.map;
            return true;
        }
    const PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return false;
    CUtensorMap map;
    const cuuint64_t dims[2] = {cuuint64_t(m), cuuint64_t(n)};
    const cuuint64_t strides[1] = {cuuint64_t(m) * sizeof(double)};
    const cuuint32_t box[2] = {uint32_t(PTileStage::W), uint32_t(PTileStage::H)};
    const cuuint32_t es[2] = {1, 1};
    CUresult r = encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(p), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    if (cache.size() >= 256) cache.erase(cache.begin());
    cache.push_back(Entry{p, m, n, map});
    *out = map;
    return true;
}

/** The persistent tile's shared-memory opt-in, set once per instantiation. */
template <int MODE, typename TC>
static bool ptile_attr() {
    static int state = -1;
    if (state < 0) {
        state = cudaFuncSetAttribute(cc_ptile<MODE, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(PTileStage::SMEM)) == cudaSuccess;
        if (!state) cudaGetLastError();
    }
    return state == 1;
}

/** The one-time setup of the persistent tile, done when a hierarchy is
 * created so that no lookup happens while a solve is being captured. */
static void ptile_prepare() {
    (void)tensor_map_encoder();
    (void)ptile_attr<0, double>();
    (void)ptile_attr<1, double>();
    (void)ptile_attr<0, float>();
    (void)ptile_attr<1, float>();
}

static int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            n = 148;
    }
    return n;
}

/** The persistent TMA-fed tile for an FP64 cell-centred level; false when it
 * does not apply (the caller then launches another tile kernel). */
template <int MODE, typename TC>
static bool launch_cc_ptile(cudaStream_t s, const CCc<double>& c, const TileArgs<double, TC>& a) {
    CUtensorMap mz, mb;
    const bool read_z = MODE == 1 || !a.zero_init;
    if (!tile_tensor_map(a.b, c.m, c.n, &mb)) return false;
    if (read_z) {
        if (!tile_tensor_map(a.zin, c.m, c.n, &mz)) return false;
    } else {
        mz = mb;   // not read
    }
    if (!ptile_attr<MODE, TC>()) return false;
    using G = CCReg<double>;
    const int nwx = (c.m + G::TX - 1) / G::TX, nwy = (c.n + G::TY - 1) / G::TY, nwin = nwx * nwy;
    const int grid = std::min(nwin, sm_count());
    cc_ptile<MODE, TC><<<grid, G::NT, PTileStage::SMEM, s>>>(c, a, mz, mb, nwx, nwin);
    g_ptile_launches.fetch_add(1, std::memory_order_relaxed);
    return true;
}

template <typename T, int MODE, typename TC = T>
static void launch_cc_tile(cudaStream_t s, const CCc<T>& c, const TileArgs<T, TC>& a) {
    if constexpr (std::is_same<T, double>::value) {
        if (reg_tile_mode() == 3 && launch_cc_ptile<MODE, TC>(s, c, a)) return;
    }
    if (use_reg_tile()) {
        using G = CCReg<T>;
        dim3 grid((c.m + G::TX - 1) / G::TX, (c.n + G::TY - 1) / G::TY);
        if (reg_tile_mode() == 2) cc_rtile<T, MODE, TC, 1><<<grid, G::NT, 0, s>>>(c, a);
        else cc_rtile<T, MODE, TC, 2><<<grid, G::NT, 0, s>>>(c, a);
        return;
    }
    using G = CCTile<T, 2>;
    dim3 grid((c.m + G::TX - 1) / G::TX, (c.n + G::TY - 1) / G::TY);
    cc_tile<T, MODE, 2, TC><<<grid, G::NT, G::smem, s>>>(c, a);
}

template <typename T, int MODE, typename TC = T>
static void launch_fem_tile(cudaStream_t s, const FEMc<T>& c, const TileArgs<T, TC>& a) {
    if (use_reg_tile()) {
        using G = FEMReg<T>;
        dim3 grid((c.M + G::TX - 1) / G::TX, (c.N + G::TY - 1) / G::TY);
        if (reg_tile_mode() == 2) fem_rtile<T, MODE, TC, 1><<<grid, G::NT, 0, s>>>(c, a);
        else fem_rtile<T, MODE, TC, 2><<<grid, G::NT, 0, s>>>(c, a);
        return;
    }
    using G = FEMTile<T>;
    dim3 grid((c.M + G::TX - 1) / G::TX, (c.N + G::TY - 1) / G::TY);
    fem_tile<T, MODE, TC><<<grid, G::NT, G::smem, s>>>(c, a);
}

template <typename T, typename TC = T>
static cudaError_t fem_tile_attr() {
    using G = FEMTile<T>;
    cudaError_t e = cudaFuncSetAttribute(fem_tile<T, 0, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(G::smem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(fem_tile<T, 1, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(G::smem));
}

template <typename T, typename TC = T>
static cudaError_t cc_tile_attr() {
    using G = CCTile<T, 2>;
    cudaError_t e = cudaFuncSetAttribute(cc_tile<T, 0, 2, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(G::smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(cc_tile<T, 1, 2, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(G::smem));
    return e;
}

/** *out = mean of x (deterministic grid reduction in FP64). */
__global__ void mean_k(const double* __restrict__ x, long N, Reduce rd, double* out) {
    double s = 0;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < N; k += long(gridDim.x) * blockDim.x) s += x[k];
    s = block_sum(s);
    double total;
    if (grid_sum(s, rd, &total) && threadIdx.x == 0) *out = total / double(N);
}

__global__ void sub_mean_k(const double* src, double* dst, long N, const double* __restrict__ mean) {
    const double mu = *mean;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < N; k += long(gridDim.x) * blockDim.x)
        dst[k] = src[k] - mu;
}

#include "mg_general.cuh"
#include "mg_cluster.cuh"
#include "mg_fast.cuh"

class MG {
  public:
    int kind = 0;
    int m = 0, n = 0;      // fine grid of the problem class (cells or nodes)
    double c1 = 0, c2 = 0; // xxsp,yysp (MAC), dx,dy (FEM) or vfx,vfy (viscous)
    int x_sym = 0;
    std::vector<LevelD> lv;
    FEMOp fop{};
    int nlev = 0;
    int nmulti64 = 0, nmulti32 = 0;
    // the coarsest level is solved by tile smoothing instead of the CTA cycle
    bool smooth_tail = false;
    size_t smem64 = 0, smem32 = 0;
    // device buffers: index l holds level l (level 0 of z64/b64 is the caller's)
    std::vector<double*> z64, b64, t64;
    std::vector<float*> z32, b32, t32;   // t: scratch iterate of each tiled level
    Reduce rd;
    SolveCtl* ctl = nullptr;
    // grids the constant-stencil hierarchy cannot coarsen use the Galerkin
    // hierarchy of mg_general.cuh (FP64 only)
    bool general = false;
    GenMG gen;
    // levels whose arrays fit in this many bytes run in the single-CTA cycle
    // (autotuned per grid; at most CTA_SMEM_LIMIT)
    size_t cta_limit = CTA_SMEM_LIMIT;
    // the first CTA-resident level with at most DIRECT_MAX unknowns is solved
    // exactly with its inverse instead of by the coarser levels' smoothing
    int dlev = -1;
    double* dinv64 = nullptr;
    float* dinv32 = nullptr;
    // the level solved exactly over the whole GPU (GDIRECT_MAX; FEM by
    // default, cell-centred systems with VDI_MG_MAC_DIRECT=1), or -1; both
    // precisions' V-cycles then stop there
    int gdlev = -1;
    double* gdinv64 = nullptr;
    float* gdinv32 = nullptr;
    int gdpitch = 0;             // their row pitch
    bool allow_gdirect = true;   // false where the inverse would need an allocation
    // the level solved exactly by the separable transform solve, or -1
    int fclev = -1, fc_j0 = 0, fc_rp = 0, fc_steps = 0;
    FastArrays<double> fc64;
    FastArrays<float> fc32;
    bool allow_fast = true;      // false where its arrays would need an allocation
    // the cluster-resident coarse cycle (mg_cluster.cuh) of the FP64 and FP32
    // V-cycles: its top level (-1: not used), CTAs and shared memory per CTA
    struct ClusterPlan {
        int top = -1, cs = 0;
        size_t smem = 0;
    };
    ClusterPlan cl64, cl32;
    bool allow_cluster = true;   // false where the exact coarsest level cannot be set up
    int nu1 = 2, nu2 = 2;
    double rtol = 1e-10;
    int max_it = 200;

    ~MG() { release(); }

    void release() {
        for (auto p : z64) if (p) cudaFree(p);
        for (auto p : b64) if (p) cudaFree(p);
        for (auto p : z32) if (p) cudaFree(p);
        for (auto p : b32) if (p) cudaFree(p);
        for (auto p : t64) if (p) cudaFree(p);
        for (auto p : t32) if (p) cudaFree(p);
        z64.clear(); b64.clear(); z32.clear(); b32.clear(); t64.clear(); t32.clear();
        reduce_free(rd);
        if (ctl) cudaFree(ctl);
        ctl = nullptr;
        gen.release();
        if (dinv64) cudaFree(dinv64);
        if (dinv32) cudaFree(dinv32);
        dinv64 = nullptr;
        dinv32 = nullptr;
        dlev = -1;
        free_gdirect();
        free_fast();
        if (bproj) cudaFree(bproj);
        if (dmean) cudaFree(dmean);
        bproj = nullptr;
        dmean = nullptr;
    }

    void free_fast() {
        fc64.release();
        fc32.release();
        fclev = -1;
    }
    const FastArrays<double>& fcarr(double*) const { return fc64; }
    const FastArrays<float>& fcarr(float*) const { return fc32; }

    void free_gdirect() {
        if (gdinv64) cudaFree(gdinv64);
        if (gdinv32) cudaFree(gdinv32);
        gdinv64 = nullptr;
        gdinv32 = nullptr;
        gdlev = -1;
    }

    bool fem() const { return kind == VDI_MG_FEM; }
    bool mac_like() const { return kind == VDI_MG_MAC || kind == VDI_MG_MAC_NEUMANN; }
    /** The pure-Neumann variant: singular (constants), solved on the
     * zero-mean part of the source, with a zero-mean solution. */
    bool neumann() const { return kind == VDI_MG_MAC_NEUMANN; }
    double* bproj = nullptr;   // the source minus its mean (Neumann variant)
    double* dmean = nullptr;   // a mean computed on the device
    /** The source the iterations use. */
    const double* rhs(const double* b) const { return neumann() ? bproj : b; }
    long size(int l) const { return long(lv[l].m) * lv[l].n; }

    /** Diagonals and couplings of level l, matching the problem classes'
     * a_cc / mul_a (mgs_mac.hh:33-45, visco_impl.hh:36-46) with the level's
     * scaled coefficients. */
    void fill_cc(LevelD& L, double kx, double ky) {
        L.ox = mac_like() ? kx : -kx;
        L.oy = mac_like() ? ky : -ky;
        bool horiz = kind == VDI_MG_VISC_U;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                double v;
                if (mac_like()) {
                    double xp = a == 1 ? -2 * kx : -kx;
                    double yp = b == 0 ? (neumann() ? -ky : -3 * ky) : (b == 1 ? -2 * ky : -ky);
                    v = xp + yp;
                } else {
                    double yp = b == 0 ? ky : 2 * ky;
                    if (x_sym) {
                        double xp = a == 0 ? (horiz ? 3 * kx : kx) : 2 * kx;
                        v = 1 + xp + yp;
                    } else {
                        v = 1 + 2 * kx + yp;
                    }
                }
                L.d[a][b] = v;
            }
        if (mac_like()) {
            L.gL = 1; L.gR = 1; L.gD = neumann() ? 1 : -1; L.gU = 1;
        } else {
            L.gL = x_sym ? (horiz ? -1 : 1) : 0;
            L.gR = 0; L.gD = 1; L.gU = 0;
        }
    }

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

    /** Chooses the hierarchy: the constant-stencil one when it reaches a
     * small coarsest level (or, for the viscous systems, one weakly coupled
     * enough for smoothing alone), the general one otherwise or when
     * VDI_MG_GENERAL is set. */
    int build_levels() {
        general = false;
        const char* e = getenv("VDI_MG_GENERAL");
        int st = build_fast_levels();
        bool need = (e && atoi(e) != 0) || st != VDI_OK;
        if (!need) {
            const LevelD& C = lv.back();
            bool small = size(nlev - 1) <= 64;
            bool weak = !mac_like() && kind != VDI_MG_FEM && 2 * (std::fabs(C.ox) + std::fabs(C.oy)) < 0.25;
            need = !small && !weak;
        }
        if (!need) return VDI_OK;
        lv.resize(1);
        if (fem()) fill_fem(lv[0]);
        else fill_cc(lv[0], c1, c2);
        nlev = 1;
        nmulti64 = nmulti32 = 0;
        smooth_tail = false;
        smem64 = smem32 = 0;
        cl64 = cl32 = ClusterPlan{};
        general = true;
        return VDI_OK;
    }

    int build_fast_levels() {
        lv.clear();
        cl64 = cl32 = ClusterPlan{};
        if (fem()) {
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
            double kx = c1, ky = c2;   // MAC: xxsp, yysp; viscous: vfx, vfy
            int mm = m, nn = n;
            while (true) {
                LevelD L{};
                L.m = mm; L.n = nn;
                fill_cc(L, kx, ky);
                lv.push_back(L);
                if ((mm & 1) || (nn & 1) || mm < 4 || nn < 2 || int(lv.size()) == MAXLEV) break;
                // The viscous operator I - vfx Dxx - vfy Dyy is close to the
                // identity once 2(vfx+vfy) is small: Gauss-Seidel alone solves
                // that level, and coarser levels add nothing.
                if (!mac_like() && lv.size() >= 2 && 2 * (kx + ky) < 0.25) break;
                mm >>= 1; nn >>= 1;
                kx *= 0.25; ky *= 0.25;
            }
        }
        nlev = int(lv.size());
        smooth_tail = kind == VDI_MG_VISC_U || kind == VDI_MG_VISC_V;
        if (smooth_tail) {
            if (nlev < 2) {
                set_error("multigrid: viscous %dx%d grid cannot coarsen", m, n);
                return VDI_ERR_UNSUPPORTED_SIZE;
            }
            nmulti64 = nmulti32 = nlev - 1;
            smem64 = smem32 = 0;
            return VDI_OK;
        }
        // the CTA-resident tail must fit in shared memory
        int arrays = fem() ? 3 : 2;
        auto tail_bytes = [&](int from, size_t es) {
            size_t t = 0;
            for (int l = from; l < nlev; l++) t += size_t(arrays) * size(l) * es;
            return t;
        };
        nmulti64 = -1;
        for (int l = 0; l < nlev; l++)
            if (tail_bytes(l, 8) <= cta_limit) { nmulti64 = l; break; }
        nmulti32 = -1;
        for (int l = 0; l < nlev; l++)
            if (tail_bytes(l, 4) <= cta_limit) { nmulti32 = l; break; }
        if (nmulti64 < 0 || nmulti32 < 0) {
            set_error("multigrid: %dx%d grid does not coarsen to a shared-memory-sized level", m, n);
            return VDI_ERR_UNSUPPORTED_SIZE;
        }
        smem64 = tail_bytes(nmulti64, 8);
        smem32 = tail_bytes(nmulti32, 4);
        cl64 = plan_cluster<double>();
        cl32 = plan_cluster<float>();
        if (cl64.top >= 0) nmulti64 = cl64.top;
        if (cl32.top >= 0) nmulti32 = cl32.top;
        free_gdirect();
        free_fast();
        if (setup_fast() == VDI_OK && fclev >= 0) {
            nmulti32 = nmulti64 = fclev;
            cl64 = cl32 = ClusterPlan{};
        } else if (setup_gdirect() == VDI_OK && gdlev >= 0) {
            nmulti32 = nmulti64 = gdlev;
            cl64 = cl32 = ClusterPlan{};
        }
        return VDI_OK;
    }

    /** Shared-memory layout of the cluster cycle from level `top` (cs CTAs):
     * fills a when given; returns the elements per CTA. */
    template <typename T>
    long cluster_layout(int top, int cs, int dl, CCClusterArgs<T>* a) const {
        long off = 0;
        for (int q = 0; top + q < dl; q++) {
            const int l = top + q;
            const long mm = lv[l].m, h = lv[l].n / cs;
            if (a) {
                a->lv[q] = ccc<T>(l);
                a->h[q] = int(h);
                a->oz[q] = int(off);
                a->ob[q] = int(off + (h + 2 * CL_G) * mm);
                a->opre[q] = int(off + 2 * (h + 2 * CL_G) * mm);
                a->opost[q] = int(off + 2 * (h + 2 * CL_G) * mm + 8 * mm);
            }
            off += 2 * (h + 2 * CL_G) * mm + 8 * mm + (q > 0 ? 6 * mm : 0);
        }
        if (a) {
            a->nd = dl - top;
            a->cs = cs;
            a->dl = ccc<T>(dl);
            a->ostage = int(off);
        }
        off += size(dl - 1);
        if (a) a->odb = int(off);
        off += size(dl);
        if (a) a->odz = int(off);
        off += size(dl);
        return off;
    }

    /** The cluster cycle for this hierarchy, if it applies: cell-centred
     * systems with an exact coarsest level whose finer neighbour splits into
     * equal row slabs; the top level is the finest whose slabs fit in shared
     * memory. VDI_MG_CLUSTER=0 turns it off. */
    template <typename T>
    ClusterPlan plan_cluster() const {
        ClusterPlan p;
        const char* e = getenv("VDI_MG_CLUSTER");
        if ((e && atoi(e) == 0) || !allow_cluster || fem() || smooth_tail || neumann() || general) return p;
        int dl = -1;
        for (int l = 0; l < nlev; l++)
            if (size(l) <= DIRECT_MAX) {
                dl = l;
                break;
            }
        if (dl < 1) return p;
        if (cc_cluster_attr<T>() != cudaSuccess) {
            cudaGetLastError();
            return p;
        }
        for (int cs : {16, 8}) {
            if (lv[dl - 1].n % cs) continue;
            for (int top = std::max(0, dl - CL_MAXLEV); top < dl; top++) {
                // a thread owns one column of the widest slab level
                if (lv[top].m > CL_THREADS) continue;
                const size_t bytes = size_t(cluster_layout<T>(top, cs, dl, nullptr)) * sizeof(T);
                if (bytes > CL_SMEM_LIMIT) continue;
                if (cc_cluster_fits<T>(cs, bytes) <= 0) break;
                p.top = top;
                p.cs = cs;
                p.smem = bytes;
                return p;
            }
        }
        return p;
    }
    const ClusterPlan& cplan(double*) const { return cl64; }
    const ClusterPlan& cplan(float*) const { return cl32; }

    int alloc() {
        if (neumann()) {
            VDI_CUDA(cudaMalloc(&bproj, size(0) * sizeof(double)));
            VDI_CUDA(cudaMalloc(&dmean, sizeof(double)));
        }
        if (general) {
            VDI_TRY(reduce_alloc(rd, MAX_PARTIALS));
            VDI_CUDA(cudaMalloc(&ctl, sizeof(SolveCtl)));
            VDI_CUDA(cudaMemset(ctl, 0, sizeof(SolveCtl)));
            VDI_TRY(set_ctl_params(0, rtol, max_it));
            const long N0 = size(0);
            auto apply = [&](const double* z, double* y) -> int {
                if (fem()) apply_k<double><<<nblk(N0), 256>>>(femc<double>(0), z, y);
                else apply_k<double><<<nblk(N0), 256>>>(ccc<double>(0), z, y);
                VDI_CUDA(cudaGetLastError());
                return VDI_OK;
            };
            VDI_TRY(gen.setup(m, n, apply, neumann()));
            VDI_CUDA(cudaDeviceSynchronize());
            return VDI_OK;
        }
        z64.assign(nlev, nullptr); b64.assign(nlev, nullptr);
        z32.assign(nlev, nullptr); b32.assign(nlev, nullptr);
        t64.assign(nlev, nullptr); t32.assign(nlev, nullptr);
        for (int l = 0; l < nlev; l++) {
            size_t s = size_t(size(l));
            if (l < nmulti64) VDI_CUDA(cudaMalloc(&t64[l], s * 8));
            if (l < nmulti32) VDI_CUDA(cudaMalloc(&t32[l], s * 4));
            if (l > 0 && l <= nmulti64) {
                VDI_CUDA(cudaMalloc(&z64[l], s * 8));
                VDI_CUDA(cudaMalloc(&b64[l], s * 8));
            }
            if (l <= nmulti32) {
                VDI_CUDA(cudaMalloc(&z32[l], s * 4));
                VDI_CUDA(cudaMalloc(&b32[l], s * 4));
            }
        }
        VDI_TRY(reduce_alloc(rd, MAX_PARTIALS));
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
        VDI_CUDA(cc_tile_attr<double>());
        VDI_CUDA(cc_tile_attr<float>());
        VDI_CUDA((cc_tile_attr<double, float>()));
        VDI_CUDA(fem_tile_attr<double>());
        VDI_CUDA(fem_tile_attr<float>());
        VDI_CUDA((fem_tile_attr<double, float>()));
        VDI_TRY(setup_direct());
        return VDI_OK;
    }

    /** Sweeps on the coarsest level: enough for its few points, few enough
     * that the single-CTA cycle stays short. */
    int ncoarse_sweeps() const {
        int s = lv[nlev - 1].m + lv[nlev - 1].n;
        return std::min(32, std::max(4, s));
    }

    template <typename T>
    TileArgs<T> targs(const T* zin, T* zout, const T* b) const {
        TileArgs<T> a{};
        a.zin = zin;
        a.zout = zout;
        a.b = b;
        a.rd = rd;
        a.ctl = ctl;
        return a;
    }

    const double* dinv(double*) const { return dinv64; }
    const float* dinv(float*) const { return dinv32; }

    /** The separable exact solve (mg_fast.cuh) of the first level with at
     * most FAST_MAX unknowns, when the operator there is separable in the
     * cosine basis of its centring (VDI_MG_FAST_COARSE=0 turns it off). A
     * solve of a random source is checked against the operator before it is
     * used; any failure leaves the other coarse paths. */
    int setup_fast() {
        const char* e = getenv("VDI_MG_FAST_COARSE");
        if ((e && atoi(e) == 0) || !allow_fast || general || smooth_tail || neumann()) return VDI_OK;
        // VDI_MG_FAST_MAX overrides the size bound (measurements)
        const char* em = getenv("VDI_MG_FAST_MAX");
        const long fmax = em && atol(em) > 0 ? atol(em) : FAST_MAX;
        int l = -1;
        for (int q = 1; q < nlev && l < 0; q++)
            if (size(q) <= fmax) l = q;
        if (l < 0) return VDI_OK;
        const int ml = lv[l].m, nl = lv[l].n;
        const long N = size(l);
        if (ml > 2048) return VDI_OK;   // bounds the two m x m basis matrices
        double *S = nullptr, *zt = nullptr, *bt = nullptr, *yt = nullptr;
        auto done = [&](int code) {
            cudaGetLastError();
            for (double* p : {S, zt, bt, yt})
                if (p) cudaFree(p);
            if (fclev < 0) {
                fc64.release();
                fc32.release();
            }
            return code;
        };
        if (cudaMalloc(&S, 9 * N * sizeof(double)) != cudaSuccess) return done(VDI_ERR_CUDA);
        auto apply = [&](const double* z, double* y) -> int {
            if (fem()) apply_k<double><<<nblk(N), 256>>>(femc<double>(l), z, y);
            else apply_k<double><<<nblk(N), 256>>>(ccc<double>(l), z, y);
            VDI_CUDA(cudaGetLastError());
            return VDI_OK;
        };
        if (probe_stencil(ml, nl, S, apply) != VDI_OK) return done(VDI_OK);
        std::vector<double> Sh(9 * size_t(N));
        if (cudaMemcpy(Sh.data(), S, Sh.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return done(VDI_ERR_CUDA);
        FastHost F;
        if (!fast_analyse(Sh, ml, nl, fem(), F)) return done(VDI_OK);
        if (fast_upload<double>(F, fc64) != VDI_OK || fast_upload<float>(F, fc32) != VDI_OK) return done(VDI_ERR_CUDA);
        // check: A (A^-1 b) = b for a pseudo-random source
        std::vector<double> bh(N), yh(N);
        unsigned r = 12345u;
        for (long k = 0; k < N; k++) {
            r = r * 1664525u + 1013904223u;
            bh[k] = double(r >> 8) / double(1u << 24) - 0.5;
        }
        if (cudaMalloc(&zt, N * sizeof(double)) != cudaSuccess || cudaMalloc(&bt, N * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&yt, N * sizeof(double)) != cudaSuccess ||
            cudaMemcpy(bt, bh.data(), N * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
            return done(VDI_ERR_CUDA);
        if (fast_solve<double>(0, fc64, ml, nl, F.j0, F.rp, F.steps, bt, zt) != VDI_OK || apply(zt, yt) != VDI_OK ||
            cudaMemcpy(yh.data(), yt, N * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return done(VDI_ERR_CUDA);
        double err = 0, bmax = 0;
        for (long k = 0; k < N; k++) {
            err = std::max(err, std::fabs(yh[k] - bh[k]));
            bmax = std::max(bmax, std::fabs(bh[k]));
        }
        if (!(err <= 1e-10 * bmax)) return done(VDI_OK);
        fclev = l;
        fc_j0 = F.j0;
        fc_rp = F.rp;
        fc_steps = F.steps;
        return done(VDI_OK);
    }

    /** The whole-GPU exact solve of a FEM hierarchy's first CTA-resident
     * level, when it has more than DIRECT_MAX and at most GDIRECT_MAX
     * unknowns (VDI_MG_FEM_DIRECT=0 turns it off): the level's operator is
     * probed into a stencil and inverted on the device. A failed inversion
     * leaves the single-CTA cycle in place. */
    int setup_gdirect() {
        if (!allow_gdirect || general || smooth_tail || neumann()) return VDI_OK;
        int l = -1;
        if (fem()) {
            const char* e = getenv("VDI_MG_FEM_DIRECT");
            if ((e && atoi(e) == 0) || nmulti64 < 1) return VDI_OK;
            l = nmulti64;
        } else {
            // cell-centred: opt-in (VDI_MG_MAC_DIRECT=1), the first level
            // small enough, in place of the cluster or single-CTA cycle
            const char* e = getenv("VDI_MG_MAC_DIRECT");
            if (!e || atoi(e) == 0) return VDI_OK;
            for (int q = 1; q < nlev && l < 0; q++)
                if (size(q) <= GDIRECT_MAX) l = q;
            if (l < 0) return VDI_OK;
        }
        const long N = size(l);
        if (N <= DIRECT_MAX || N > GDIRECT_MAX) return VDI_OK;
        const int ml = lv[l].m, nl = lv[l].n;
        double *S = nullptr, *A = nullptr, *rk = nullptr, *ck = nullptr;
        int* bad = nullptr;
        int st = VDI_OK;
        auto fail = [&](int code) {
            cudaGetLastError();
            if (S) cudaFree(S);
            if (A) cudaFree(A);
            if (rk) cudaFree(rk);
            if (ck) cudaFree(ck);
            if (bad) cudaFree(bad);
            return code;
        };
        if (cudaMalloc(&S, 9 * N * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&A, size_t(N) * N * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&rk, N * sizeof(double)) != cudaSuccess || cudaMalloc(&ck, N * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&bad, sizeof(int)) != cudaSuccess)
            return fail(VDI_ERR_CUDA);
        auto apply = [&](const double* z, double* y) -> int {
            if (fem()) apply_k<double><<<nblk(N), 256>>>(femc<double>(l), z, y);
            else apply_k<double><<<nblk(N), 256>>>(ccc<double>(l), z, y);
            VDI_CUDA(cudaGetLastError());
            return VDI_OK;
        };
        st = probe_stencil(ml, nl, S, apply);
        if (st != VDI_OK) return fail(st);
        if (cudaMemset(A, 0, size_t(N) * N * sizeof(double)) != cudaSuccess ||
            cudaMemset(bad, 0, sizeof(int)) != cudaSuccess)
            return fail(VDI_ERR_CUDA);
        const int nb = int((N + 255) / 256);
        gj_assemble_k<<<nb, 256>>>(S, ml, nl, A);
        for (int k = 0; k < N; k++) {
            gj_pivot_k<<<nb, 256>>>(A, int(N), k, rk, ck, bad);
            gj_update_k<<<dim3(nb, unsigned(N)), 256>>>(A, int(N), k, rk, ck);
        }
        int hbad = 0;
        if (cudaMemcpy(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return fail(VDI_ERR_CUDA);
        if (hbad) return fail(VDI_OK);   // a zero pivot: keep the CTA cycle
        // rows padded to a multiple of 4 elements for 16-byte loads
        const int P = int((N + 3) & ~3L);
        double* X64 = nullptr;
        float* X32 = nullptr;
        if (cudaMalloc(&X64, size_t(N) * P * sizeof(double)) != cudaSuccess) return fail(VDI_ERR_CUDA);
        if (cudaMalloc(&X32, size_t(N) * P * sizeof(float)) != cudaSuccess) {
            cudaFree(X64);
            return fail(VDI_ERR_CUDA);
        }
        pad_rows_k<<<std::min(nblk(long(N) * P), 4096), 256>>>(A, int(N), P, X64, X32);
        if (cudaDeviceSynchronize() != cudaSuccess) {
            cudaFree(X64);
            cudaFree(X32);
            return fail(VDI_ERR_CUDA);
        }
        gdinv64 = X64;
        gdinv32 = X32;
        gdpitch = P;
        gdlev = l;
        return fail(VDI_OK);   // frees the scratch
    }
    const double* gdinv(double*) const { return gdinv64; }
    const float* gdinv(float*) const { return gdinv32; }

    /** The direct coarsest solve: the first CTA-resident level with at most
     * DIRECT_MAX unknowns, its operator probed into a stencil and inverted. */
    int setup_direct() {
        if (smooth_tail || general || neumann()) return VDI_OK;
        for (int l = 0; l < nlev; l++)
            if (size(l) <= DIRECT_MAX) {
                dlev = l;
                break;
            }
        if (dlev < 0) return VDI_OK;
        const int ml = lv[dlev].m, nl = lv[dlev].n;
        const long N = size(dlev);
        double* S;
        VDI_CUDA(cudaMalloc(&S, 9 * N * sizeof(double)));
        const int d = dlev;
        auto apply = [&](const double* z, double* y) -> int {
            if (fem()) apply_k<double><<<nblk(N), 256>>>(femc<double>(d), z, y);
            else apply_k<double><<<nblk(N), 256>>>(ccc<double>(d), z, y);
            VDI_CUDA(cudaGetLastError());
            return VDI_OK;
        };
        int st = probe_stencil(ml, nl, S, apply);
        std::vector<double> X;
        if (st == VDI_OK) st = stencil_inverse(S, ml, nl, X);
        cudaFree(S);
        if (st != VDI_OK) {
            dlev = -1;
            return st;
        }
        std::vector<float> Xf(X.begin(), X.end());
        VDI_CUDA(cudaMalloc(&dinv64, X.size() * sizeof(double)));
        VDI_CUDA(cudaMalloc(&dinv32, X.size() * sizeof(float)));
        VDI_CUDA(cudaMemcpy(dinv64, X.data(), X.size() * sizeof(double), cudaMemcpyHostToDevice));
        VDI_CUDA(cudaMemcpy(dinv32, Xf.data(), Xf.size() * sizeof(float), cudaMemcpyHostToDevice));
        return VDI_OK;
    }

    double* ztmp(int l, double*) { return t64[l]; }
    float* ztmp(int l, float*) { return t32[l]; }

    /** One V-cycle from level l (precision T); z/b are level-l arrays. When
     * norm is set, level 0's POST kernel ends with the residual norm and the
     * solve decision. */
    template <typename T>
    int vcycle(cudaStream_t s, int l, const T* b, T* z, int nmulti, std::vector<T*>& zs, std::vector<T*>& bs,
               size_t smem, int zero_init, int norm, int use_cond, cudaGraphConditionalHandle h) {
        if (l == nmulti && smooth_tail) {
            TileArgs<T> a = targs<T>(nullptr, z, b);
            a.zero_init = 1;
            launch_cc_tile<T, 0>(s, ccc<T>(l), a);
            VDI_CUDA(cudaGetLastError());
            return VDI_OK;
        }
        if (l == nmulti && fclev == l)
            return fast_solve<T>(s, fcarr(static_cast<T*>(nullptr)), lv[l].m, lv[l].n, fc_j0, fc_rp, fc_steps, b, z);
        if (l == nmulti && gdlev == l) {
            const int N = int(size(l));
            direct_matvec_k<T><<<(N + 7) / 8, 256, size_t(gdpitch) * sizeof(T), s>>>(
                gdinv(static_cast<T*>(nullptr)), N, gdpitch, b, z);
            VDI_CUDA(cudaGetLastError());
            return VDI_OK;
        }
        if (l == nmulti && cplan(static_cast<T*>(nullptr)).top == l) {
            const ClusterPlan& cp = cplan(static_cast<T*>(nullptr));
            if (dlev < 0 || !dinv(static_cast<T*>(nullptr))) {
                set_error("multigrid: the cluster cycle needs the exact coarsest level");
                return VDI_ERR_CUDA;
            }
            CCClusterArgs<T> a{};
            cluster_layout<T>(l, cp.cs, dlev, &a);
            a.dinv = dinv(static_cast<T*>(nullptr));
            return launch_cc_cluster<T>(s, a, cp.smem, b, z, zero_init);
        }
        if (l == nmulti) {
            if (fem()) {
                FEMStack<T> st{};
                st.nl = nlev - l;
                int off = 0;
                for (int q = 0; q < st.nl; q++) {
                    st.lv[q] = femc<T>(l + q);
                    st.off[q] = off;
                    off += 3 * int(size(l + q));
                }
                st.nu1 = nu1; st.nu2 = nu2; st.ncoarse = ncoarse_sweeps();
                if (dlev >= l && dinv(static_cast<T*>(nullptr))) {
                    st.nl = dlev - l + 1;
                    st.dinv = dinv(static_cast<T*>(nullptr));
                }
                fem_cta_cycle<T><<<1, CTA_THREADS, smem, s>>>(st, b, z, zero_init);
            } else {
                CCStack<T> st{};
                st.nl = nlev - l;
                int off = 0;
                for (int q = 0; q < st.nl; q++) {
                    st.lv[q] = ccc<T>(l + q);
                    st.off[q] = off;
                    off += 2 * int(size(l + q));
                }
                st.nu1 = nu1; st.nu2 = nu2; st.ncoarse = ncoarse_sweeps();
                if (dlev >= l && dinv(static_cast<T*>(nullptr))) {
                    st.nl = dlev - l + 1;
                    st.dinv = dinv(static_cast<T*>(nullptr));
                }
                cc_cta_cycle<T><<<1, CTA_THREADS, smem, s>>>(st, b, z, zero_init);
            }
            VDI_CUDA(cudaGetLastError());
            return VDI_OK;
        }
        // PRE writes the level's scratch iterate, POST reads it and writes z
        T* zs_tmp = ztmp(l, static_cast<T*>(nullptr));
        TileArgs<T> a = targs<T>(z, zs_tmp, b);
        a.zero_init = zero_init;
        a.bc = bs[l + 1];
        if (fem()) launch_fem_tile<T, 0>(s, femc<T>(l), a);
        else launch_cc_tile<T, 0>(s, ccc<T>(l), a);
        VDI_CUDA(cudaGetLastError());
        VDI_TRY(vcycle<T>(s, l + 1, bs[l + 1], zs[l + 1], nmulti, zs, bs, smem, 1, 0, 0, 0));
        TileArgs<T> p = targs<T>(zs_tmp, z, b);
        p.zc = zs[l + 1];
        p.norm = norm;
        p.use_cond = use_cond;
        p.h = h;
        if (fem()) launch_fem_tile<T, 1>(s, femc<T>(l), p);
        else launch_cc_tile<T, 1>(s, ccc<T>(l), p);
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    int vcycle64(cudaStream_t s, const double* b, double* z, int norm, int use_cond, cudaGraphConditionalHandle h) {
        if (general) {
            VDI_TRY(gen.vcycle(s, 0, b, z));
            if (norm) VDI_TRY(enqueue_resid_norm(s, b, z, 1, use_cond, h));
            return VDI_OK;
        }
        VDI_TRY(vcycle<double>(s, 0, b, z, nmulti64, z64, b64, smem64, 0, norm && nmulti64 > 0, use_cond, h));
        if (norm && nmulti64 == 0) VDI_TRY(enqueue_resid_norm(s, b, z, 1, use_cond, h));
        return VDI_OK;
    }
    /** FP64 finest level (its smoothing, residual and norm) over FP32 coarse
     * levels: the coarse-grid correction only has to be approximate, so its
     * precision does not limit the FP64 residual the loop stops on. */
    int vcycle_hybrid(cudaStream_t s, const double* b, double* z, int norm, int use_cond,
                      cudaGraphConditionalHandle h) {
        if (general || nmulti64 < 1 || nmulti32 < 1) return vcycle64(s, b, z, norm, use_cond, h);
        TileArgs<double, float> a{};
        a.zin = z;
        a.zout = t64[0];
        a.b = b;
        a.bc = b32[1];
        a.rd = rd;
        a.ctl = ctl;
        if (fem()) launch_fem_tile<double, 0, float>(s, femc<double>(0), a);
        else launch_cc_tile<double, 0, float>(s, ccc<double>(0), a);
        VDI_CUDA(cudaGetLastError());
        VDI_TRY(vcycle<float>(s, 1, b32[1], z32[1], nmulti32, z32, b32, smem32, 1, 0, 0, 0));
        TileArgs<double, float> p{};
        p.zin = t64[0];
        p.zout = z;
        p.b = b;
        p.zc = z32[1];
        p.rd = rd;
        p.ctl = ctl;
        p.norm = norm;
        p.use_cond = use_cond;
        p.h = h;
        if (fem()) launch_fem_tile<double, 1, float>(s, femc<double>(0), p);
        else launch_cc_tile<double, 1, float>(s, ccc<double>(0), p);
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    int vcycle32(cudaStream_t s) {
        return vcycle<float>(s, 0, b32[0], z32[0], nmulti32, z32, b32, smem32, 1, 0, 0, 0);
    }

    /** sblocks for the finest level. */
    int sblk0() const { return general ? sblocks(gen.gm[0], gen.gn[0]) : sblocks(lv[0].m, lv[0].n); }

    int enqueue_resid_norm(cudaStream_t s, const double* b, const double* z, int count_cycle, int use_cond,
                           cudaGraphConditionalHandle h) {
        int nb = sblk0();
        if (general)
            resid_norm_k<double><<<nb, 256, 0, s>>>(gen.op(0), z, b, rd, ctl, count_cycle, use_cond, h);
        else if (fem())
            resid_norm_k<double><<<nb, 256, 0, s>>>(femc<double>(0), z, b, rd, ctl, count_cycle, use_cond, h);
        else
            resid_norm_k<double><<<nb, 256, 0, s>>>(ccc<double>(0), z, b, rd, ctl, count_cycle, use_cond, h);
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    int enqueue_resid32(cudaStream_t s, const double* b, const double* z, int count_cycle, int use_cond,
                        cudaGraphConditionalHandle h) {
        int nb = sblk0();
        if (fem())
            resid_to32_k<<<nb, 256, 0, s>>>(femc<double>(0), z, b, b32[0], rd, ctl, count_cycle, use_cond, h);
        else
            resid_to32_k<<<nb, 256, 0, s>>>(ccc<double>(0), z, b, b32[0], rd, ctl, count_cycle, use_cond, h);
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    /** The Neumann compatibility step: dst = src - mean(src), the mean a
     * deterministic FP64 grid reduction. */
    int remove_mean(cudaStream_t s, const double* src, double* dst) {
        const long N = size(0);
        int nb = rblocks(N);
        mean_k<<<nb, 256, 0, s>>>(src, N, rd, dmean);
        sub_mean_k<<<std::min(nblk(N), 4096), 256, 0, s>>>(src, dst, N, dmean);
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    int enqueue_begin(cudaStream_t s, const double* b, double* z) {
        if (neumann()) VDI_TRY(remove_mean(s, b, bproj));
        return VDI_OK;
    }

    /** One iteration of the solve loop body (precision-dependent); ends with
     * the residual norm of the new iterate and the solve decision. */
    int enqueue_body(cudaStream_t s, const double* b, double* z, int precision, int use_cond,
                     cudaGraphConditionalHandle h) {
        if (precision == VDI_MG_HYBRID) return vcycle_hybrid(s, b, z, 1, use_cond, h);
        if (precision == VDI_MG_MIXED && !general) {
            VDI_TRY(vcycle32(s));
            if (reinterpret_cast<uintptr_t>(z) % 16 == 0)
                add_f32_to_f64_x4<<<nblk((size(0) + 3) / 4), 256, 0, s>>>(z, z32[0], size(0));
            else
                add_f32_to_f64<<<nblk(size(0)), 256, 0, s>>>(z, z32[0], size(0));
            VDI_TRY(enqueue_resid32(s, b, z, 1, use_cond, h));
        } else {
            VDI_TRY(vcycle64(s, b, z, 1, use_cond, h));
        }
        return VDI_OK;
    }

    int enqueue_first_check(cudaStream_t s, const double* b, double* z, int precision, int use_cond,
                            cudaGraphConditionalHandle h) {
        int nb = sblk0();
        if (precision == VDI_MG_MIXED && !general) {
            if (fem()) first_check_k<double><<<nb, 256, 0, s>>>(femc<double>(0), z, b, rd, ctl, use_cond, h, b32[0]);
            else first_check_k<double><<<nb, 256, 0, s>>>(ccc<double>(0), z, b, rd, ctl, use_cond, h, b32[0]);
            VDI_CUDA(cudaGetLastError());
            return VDI_OK;
        }
        if (general)
            first_check_k<double><<<nb, 256, 0, s>>>(gen.op(0), z, b, rd, ctl, use_cond, h);
        else if (fem())
            first_check_k<double><<<nb, 256, 0, s>>>(femc<double>(0), z, b, rd, ctl, use_cond, h);
        else
            first_check_k<double><<<nb, 256, 0, s>>>(ccc<double>(0), z, b, rd, ctl, use_cond, h);
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    int set_ctl_params(cudaStream_t s, double rt, int mx) {
        rtol = rt;
        max_it = mx;
        // rtol, it and max_it are consecutive in SolveCtl; write them together
        struct P {
            double rtol;
            int it;
            int max_it;
        } p{rt, 0, mx};
        static_assert(offsetof(SolveCtl, rtol) + sizeof(double) == offsetof(SolveCtl, it), "layout");
        static_assert(offsetof(SolveCtl, it) + sizeof(int) == offsetof(SolveCtl, max_it), "layout");
        VDI_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(ctl) + offsetof(SolveCtl, rtol), &p,
                                 sizeof(double) + 2 * sizeof(int), cudaMemcpyHostToDevice, s));
        VDI_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(ctl) + offsetof(SolveCtl, err_out), &err_word,
                                 sizeof(int*), cudaMemcpyHostToDevice, s));
        VDI_CUDA(cudaStreamSynchronize(s));
        return VDI_OK;
    }
    int* err_word = nullptr;   // see mg_set_error_word
};

int mg_create(int kind, int m, int n, double c1, double c2, int x_sym, MG** out) {
    if (!out || m < 2 || n < 2 || kind < 0 || kind > 4) {
        set_error("mg_create: invalid arguments");
        return VDI_ERR_INVALID_ARGUMENT;
    }
    MG* g = new MG();
    g->kind = kind; g->m = m; g->n = n; g->c1 = c1; g->c2 = c2; g->x_sym = x_sym;
    if (reg_tile_mode() == 3) ptile_prepare();
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
    // the hierarchy depth depends on vfx, vfy: rebuild it (visco_impl::setup,
    // called by setup_and_solve when vfx changes, visco_impl.cc:26-30)
    double rt = mg->rtol;
    int mx = mg->max_it;
    mg->release();
    mg->c1 = vfx;
    mg->c2 = vfy;
    mg->rtol = rt;
    mg->max_it = mx;
    VDI_TRY(mg->build_levels());
    return mg->alloc();
}

int mg_set_cta_limit(MG* mg, size_t bytes) {
    if (bytes < 1024 || bytes > CTA_SMEM_LIMIT) return VDI_ERR_INVALID_ARGUMENT;
    if (bytes == mg->cta_limit) return VDI_OK;
    double rt = mg->rtol;
    int mx = mg->max_it;
    mg->release();
    mg->cta_limit = bytes;
    mg->rtol = rt;
    mg->max_it = mx;
    VDI_TRY(mg->build_levels());
    return mg->alloc();
}

size_t mg_cta_limit(const MG* mg) { return mg->cta_limit; }
int mg_coarse_cycle(const MG* mg, int precision, int* first, int* ctas) {
    const bool f32 = precision == VDI_MG_MIXED;
    if (mg->general || mg->smooth_tail) {
        *first = -1;
        *ctas = 0;
        return VDI_OK;
    }
    const auto& cp = f32 ? mg->cl32 : mg->cl64;
    *first = f32 ? mg->nmulti32 : mg->nmulti64;
    *ctas = mg->fclev >= 0 && mg->fclev == *first ? -1
            : (mg->gdlev >= 0 && mg->gdlev == *first ? 0 : (cp.top >= 0 ? cp.cs : 1));
    return VDI_OK;
}
int mg_tiled_levels(const MG* mg, int precision) {
    if (mg->general) return -1;
    return precision == VDI_MG_MIXED ? mg->nmulti32 : mg->nmulti64;
}

SolveCtl* mg_ctl(MG* mg) { return mg->ctl; }
int mg_kind(const MG* mg) { return mg->kind; }
int mg_fine_size(const MG* mg) { return int(mg->size(0)); }
int mg_dims(const MG* mg, int* m, int* n) {
    *m = mg->m;
    *n = mg->n;
    return VDI_OK;
}

int mg_configure(MG* mg, double rtol, int max_it) { return mg->set_ctl_params(0, rtol, max_it); }
int mg_set_error_word(MG* mg, int* d_err) {
    mg->err_word = d_err;
    return mg->set_ctl_params(0, mg->rtol, mg->max_it);
}

int mg_solve(MG* mg, cudaStream_t s, const double* b, double* z, double rtol, int max_it, int precision,
             int* vcycles, double* rel_res) {
    if (rtol != mg->rtol || max_it != mg->max_it) VDI_TRY(mg->set_ctl_params(s, rtol, max_it));
    VDI_TRY(mg->enqueue_begin(s, b, z));
    const double* bb = mg->rhs(b);
    VDI_TRY(mg->enqueue_first_check(s, bb, z, precision, 0, 0));
    SolveCtl h{};
    while (true) {
        VDI_CUDA(cudaMemcpyAsync(&h, mg->ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, s));
        VDI_CUDA(cudaStreamSynchronize(s));
        if (h.done) break;
        VDI_TRY(mg->enqueue_body(s, bb, z, precision, 0, 0));
    }
    if (mg->neumann()) {
        VDI_TRY(mg->remove_mean(s, z, z));
        VDI_CUDA(cudaStreamSynchronize(s));
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
    // Loop control needs the host unless the stream is capturing, in which
    // case the loop becomes a conditional graph node.
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
    const double* bb = mg->rhs(b);
    VDI_TRY(mg->enqueue_first_check(s, bb, z, precision, 1, h));
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
    int st = mg->enqueue_body(bs, bb, z, precision, 1, h);
    cudaGraph_t bodyOut;
    e = cudaStreamEndCapture(bs, &bodyOut);
    cudaStreamDestroy(bs);
    if (st != VDI_OK) return st;
    VDI_CUDA(e);
    if (mg->neumann()) VDI_TRY(mg->remove_mean(s, z, z));
    return VDI_OK;
}

int mg_v_cycle(MG* mg, cudaStream_t s, const double* b, double* z) { return mg->vcycle64(s, b, z, 0, 0, 0); }

int mg_residual(MG* mg, cudaStream_t s, const double* b, const double* z, double* r, double* norm) {
    double* d_out;
    VDI_CUDA(cudaMallocAsync(&d_out, sizeof(double), s));
    int nb = mg->sblk0();
    if (mg->fem())
        resid_out_k<double><<<nb, 256, 0, s>>>(mg->femc<double>(0), z, b, r, mg->rd, d_out);
    else
        resid_out_k<double><<<nb, 256, 0, s>>>(mg->ccc<double>(0), z, b, r, mg->rd, d_out);
    VDI_CUDA(cudaGetLastError());
    double hn = 0;
    VDI_CUDA(cudaMemcpyAsync(&hn, d_out, sizeof(double), cudaMemcpyDeviceToHost, s));
    VDI_CUDA(cudaFreeAsync(d_out, s));
    VDI_CUDA(cudaStreamSynchronize(s));
    if (norm) *norm = hn;
    return VDI_OK;
}

int mg_kernels_per_iteration(const MG* mg, int precision) {
    if (mg->general) return mg->gen.kernels_per_vcycle() + 1;
    if (precision == VDI_MG_HYBRID) {
        if (mg->nmulti64 < 1 || mg->nmulti32 < 1) precision = VDI_MG_FP64;
        else return 2 * mg->nmulti32 + 1;
    }
    int nm = precision == VDI_MG_MIXED ? mg->nmulti32 : mg->nmulti64;
    int k = 2 * nm + 1;                       // PRE/POST per tiled level + the coarsest
    if (precision == VDI_MG_MIXED) k += 2;    // FP64 update and residual
    else if (nm == 0) k += 1;                 // separate norm when no tile level exists
    return k;
}

double mg_vcycle_bytes(const MG* mg, int fine_word, int coarse_word) {
    // canonical bytes of a V-cycle: per level, each smoothing sweep reads z
    // and b and writes z, and the transfers move 4.5 words per point
    const double per = 3. * (mg->nu1 + mg->nu2) + 4.5;
    double fine = 0, coarse = 0;
    if (mg->general) {
        for (int q = 0; q < mg->gen.nlev(); q++) (q ? coarse : fine) += double(mg->gen.size(q));
    } else {
        for (int q = 0; q < mg->nlev; q++) (q ? coarse : fine) += double(mg->size(q));
    }
    return per * (fine * fine_word + coarse * coarse_word);
}

int mg_profile(MG* mg, cudaStream_t s, int which, int iters, const double* b, double* z, float* ms, double* bytes) {
    if (iters < 1 || which < 0 || which > 6) return VDI_ERR_INVALID_ARGUMENT;
    if (which >= 4) {
        // the refinement's (mixed precision) finest kernels: 4 the FP32
        // PRE from zero, 5 the FP32 POST, 6 the FP64 residual pass that
        // writes the FP32 source and decides
        if (mg->general || mg->nmulti32 < 1) return VDI_ERR_INVALID_ARGUMENT;
        TileArgs<float> a = mg->targs<float>(which == 4 ? nullptr : mg->t32[0], which == 4 ? mg->t32[0] : mg->z32[0],
                                             mg->b32[0]);
        a.zero_init = which == 4;
        a.bc = mg->b32[1];
        a.zc = mg->z32[1];
        auto launch = [&]() -> int {
            if (which == 6) return mg->enqueue_resid32(s, b, z, 0, 0, 0);
            if (mg->fem()) {
                if (which == 4) launch_fem_tile<float, 0>(s, mg->femc<float>(0), a);
                else launch_fem_tile<float, 1>(s, mg->femc<float>(0), a);
            } else {
                if (which == 4) launch_cc_tile<float, 0>(s, mg->ccc<float>(0), a);
                else launch_cc_tile<float, 1>(s, mg->ccc<float>(0), a);
            }
            VDI_CUDA(cudaGetLastError());
            return VDI_OK;
        };
        // one refinement iteration fills the FP32 source and coarse arrays
        VDI_TRY(mg->enqueue_resid32(s, b, z, 0, 0, 0));
        VDI_TRY(mg->vcycle32(s));
        VDI_TRY(launch());
        cudaEvent_t e0, e1;
        VDI_CUDA(cudaEventCreate(&e0));
        VDI_CUDA(cudaEventCreate(&e1));
        VDI_CUDA(cudaEventRecord(e0, s));
        int st = VDI_OK;
        for (int k = 0; k < iters && st == VDI_OK; k++) st = launch();
        VDI_CUDA(cudaEventRecord(e1, s));
        VDI_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        VDI_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        VDI_TRY(st);
        *ms = t / iters;
        const double N = double(mg->size(0)), Nc = double(mg->size(1));
        // 4: b in, z out, coarse source out; 5: z, b in, z out, coarse
        // correction in (4 bytes each); 6: z, b in (8 bytes), source out (4)
        *bytes = which == 4 ? 8 * N + 4 * Nc : (which == 5 ? 12 * N + 4 * Nc : 20 * N);
        return VDI_OK;
    }
    if (which >= 2) {
        // 2: whole FP64 V-cycles back to back (mg_test.cc:36-43 times the
        // same); 3: the single-CTA coarse cycle alone
        if (which == 3 && (mg->general || mg->nmulti64 < 1 || mg->smooth_tail)) return VDI_ERR_INVALID_ARGUMENT;
        const int l = mg->nmulti64;
        auto launch = [&]() -> int {
            if (which == 2) return mg->vcycle64(s, b, z, 0, 0, 0);
            return mg->vcycle<double>(s, l, mg->b64[l], mg->z64[l], l, mg->z64, mg->b64, mg->smem64, 1, 0, 0, 0);
        };
        VDI_TRY(mg->vcycle64(s, b, z, 0, 0, 0));
        VDI_TRY(launch());
        cudaEvent_t e0, e1;
        VDI_CUDA(cudaEventCreate(&e0));
        VDI_CUDA(cudaEventCreate(&e1));
        VDI_CUDA(cudaEventRecord(e0, s));
        int st = VDI_OK;
        for (int k = 0; k < iters && st == VDI_OK; k++) st = launch();
        VDI_CUDA(cudaEventRecord(e1, s));
        VDI_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        VDI_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        VDI_TRY(st);
        *ms = t / iters;
        *bytes = which == 2 ? mg_vcycle_bytes(mg, 8, 8) : 0.;
        return VDI_OK;
    }
    if (mg->nmulti64 < 1) return VDI_ERR_INVALID_ARGUMENT;
    cudaEvent_t e0, e1;
    VDI_CUDA(cudaEventCreate(&e0));
    VDI_CUDA(cudaEventCreate(&e1));
    TileArgs<double> a = mg->targs<double>(which == 0 ? z : mg->t64[0], which == 0 ? mg->t64[0] : z, b);
    a.bc = mg->b64[1];
    a.zc = mg->z64[1];
    auto launch = [&]() {
        if (mg->fem()) {
            if (which == 0) launch_fem_tile<double, 0>(s, mg->femc<double>(0), a);
            else launch_fem_tile<double, 1>(s, mg->femc<double>(0), a);
        } else {
            if (which == 0) launch_cc_tile<double, 0>(s, mg->ccc<double>(0), a);
            else launch_cc_tile<double, 1>(s, mg->ccc<double>(0), a);
        }
    };
    // the coarse inputs of POST must hold numbers: one V-cycle fills them
    VDI_TRY(mg->vcycle64(s, b, z, 0, 0, 0));
    launch();
    VDI_CUDA(cudaEventRecord(e0, s));
    for (int k = 0; k < iters; k++) launch();
    VDI_CUDA(cudaEventRecord(e1, s));
    VDI_CUDA(cudaEventSynchronize(e1));
    float t = 0;
    VDI_CUDA(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / iters;
    // z in, b in, z out (8 bytes each per point) and the coarse array (8 bytes
    // per coarse point, written by PRE, read by POST)
    double N = double(mg->size(0)), Nc = double(mg->size(1));
    *bytes = 3 * 8 * N + 8 * Nc;
    return VDI_OK;
}

int mg_residual_async(MG* mg, cudaStream_t s, const double* b, const double* z, double* r, double* d_norm) {
    int nb = mg->sblk0();
    if (mg->fem())
        resid_out_k<double><<<nb, 256, 0, s>>>(mg->femc<double>(0), z, b, r, mg->rd, d_norm);
    else
        resid_out_k<double><<<nb, 256, 0, s>>>(mg->ccc<double>(0), z, b, r, mg->rd, d_norm);
    VDI_CUDA(cudaGetLastError());
    return VDI_OK;
}

int mg_apply(MG* mg, cudaStream_t s, const double* z, double* y) {
    long N = mg->size(0);
    if (mg->fem())
        apply_k<double><<<nblk(N), 256, 0, s>>>(mg->femc<double>(0), z, y);
    else
        apply_k<double><<<nblk(N), 256, 0, s>>>(mg->ccc<double>(0), z, y);
    VDI_CUDA(cudaGetLastError());
    return VDI_OK;
}

}  // namespace vdi

// ======================================================= allocation-free solve
// vdi_mg_solve_noalloc: an FP64 multigrid solve of the same systems as
// vdi_mg_create + vdi_mg_solve, for callers that must not allocate device
// memory: an application that owns every device allocation itself (a fixed
// memory budget or its own pool), or code that runs where an allocation
// would stall or fail (a real-time loop). Every device buffer the solve
// needs beyond the caller's b and z comes from one file-scope __device__
// array. Its hierarchy differs from the allocating one in one respect: the
// coarsest level is smoothed, not solved with a precomputed inverse (which
// would need an allocation), and the MAC cluster coarse cycle is not used;
// solves still stop on the same FP64 residual test.

namespace vdi {

/** Largest problem the allocation-free solve accepts, in unknowns (cells for
 * MAC and viscous systems, nodes for FEM). */
static constexpr long NOALLOC_MAX_UNKNOWNS = 262144;
/** Bytes of the static scratch array: the solve needs at most about
 * 16 bytes per unknown for its scratch iterates and coarse levels, plus the
 * reduction partials and control block. */
static constexpr size_t NOALLOC_SCRATCH_BYTES = 16 * size_t(NOALLOC_MAX_UNKNOWNS) + (1u << 20);

/** The scratch. It exists once on every device that loads the library and
 * lives until the process exits. Calls share it: calls that overlap on the
 * GPU (different streams, or different host threads) race on it. */
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

struct NoallocKey {
    int dev, kind, m, n, x_sym;
    double c1, c2;
    bool operator==(const NoallocKey& o) const {
        return dev == o.dev && kind == o.kind && m == o.m && n == o.n && x_sym == o.x_sym && c1 == o.c1 &&
               c2 == o.c2;
    }
};

struct NoallocEntry {
    NoallocKey key;
    MG* mg;
};

/** Hierarchies kept, least recently used first. A caller whose
 * coefficients change every call (viscous systems whose vfx, vfy follow the
 * timestep) would otherwise grow the list without bound. */
static constexpr size_t NOALLOC_CACHE_MAX = 16;

std::vector<NoallocEntry>& noalloc_cache() {
    static std::vector<NoallocEntry> c;
    return c;
}

/** Held for a whole call: the cache, the per-device base addresses and the
 * scratch array are shared by every host thread. */
std::mutex& noalloc_mutex() {
    static std::mutex mu;
    return mu;
}

/** Deletes a hierarchy whose buffers were carved from the scratch array:
 * the pointers are cleared first, so its destructor frees nothing. */
void noalloc_drop(MG* g) {
    g->z64.clear(); g->b64.clear(); g->t64.clear();
    g->ctl = nullptr;
    g->rd.partials = nullptr;
    g->rd.counter = nullptr;
    delete g;
}

/** Device address of g_noalloc_scratch on the current device, looked up once
 * per device with that device current. */
int noalloc_base(int dev, unsigned char** out) {
    static std::vector<unsigned char*> base;
    if (dev >= int(base.size())) base.resize(dev + 1, nullptr);
    if (!base[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("vdi_mg_solve_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return VDI_ERR_CUDA;
        }
        base[dev] = static_cast<unsigned char*>(p);
    }
    *out = base[dev];
    return VDI_OK;
}

/** Builds an MG whose device buffers are carved from the static scratch. */
int noalloc_build(const NoallocKey& k, unsigned char* base, MG** out) {
    MG* g = new MG();
    g->kind = k.kind; g->m = k.m; g->n = k.n; g->c1 = k.c1; g->c2 = k.c2; g->x_sym = k.x_sym;
    g->allow_cluster = false;   // its inverse would need an allocation
    g->allow_gdirect = false;   // so would this one
    g->allow_fast = false;      // and the transform solve's arrays
    int st = g->build_levels();
    if (st == VDI_OK && g->general) {
        set_error("vdi_mg_solve_noalloc: a %dx%d grid needs the general hierarchy, which allocates", k.m, k.n);
        st = VDI_ERR_UNSUPPORTED_SIZE;
    }
    if (st != VDI_OK) {
        delete g;
        return st;
    }
    size_t off = 0;
    bool fits = true;
    auto take = [&](size_t bytes) -> unsigned char* {
        off = (off + 255) & ~size_t(255);
        unsigned char* p = base + off;
        off += bytes;
        if (off > NOALLOC_SCRATCH_BYTES) fits = false;
        return p;
    };
    g->ctl = reinterpret_cast<SolveCtl*>(take(sizeof(SolveCtl)));
    g->rd.counter = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
    g->rd.partials = reinterpret_cast<double*>(take(sizeof(double) * MAX_PARTIALS));
    g->rd.max_blocks = MAX_PARTIALS;
    g->z64.assign(g->nlev, nullptr); g->b64.assign(g->nlev, nullptr); g->t64.assign(g->nlev, nullptr);
    for (int l = 0; l < g->nlev; l++) {
        size_t s = size_t(g->size(l)) * 8;
        if (l < g->nmulti64) g->t64[l] = reinterpret_cast<double*>(take(s));
        if (l > 0 && l <= g->nmulti64) {
            g->z64[l] = reinterpret_cast<double*>(take(s));
            g->b64[l] = reinterpret_cast<double*>(take(s));
        }
    }
    if (!fits) {
        set_error("vdi_mg_solve_noalloc: %dx%d needs %zu bytes of scratch, more than the %zu available", k.m, k.n,
                  off, NOALLOC_SCRATCH_BYTES);
        noalloc_drop(g);
        return VDI_ERR_UNSUPPORTED_SIZE;
    }
    // shared-memory limits of the kernels this solve launches
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(cc_cta_cycle<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   int(CTA_SMEM_LIMIT));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fem_cta_cycle<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   int(CTA_SMEM_LIMIT));
    if (e == cudaSuccess) e = cc_tile_attr<double>();
    if (e == cudaSuccess) e = fem_tile_attr<double>();
    if (e != cudaSuccess) {
        set_error("vdi_mg_solve_noalloc: %s", cudaGetErrorString(e));
        noalloc_drop(g);
        return VDI_ERR_CUDA;
    }
    *out = g;
    return VDI_OK;
}

}  // namespace
}  // namespace vdi

extern "C" int vdi_mg_solve_noalloc(int kind, int m, int n, double c1, double c2, int x_sym, const double* d_b,
                                    double* d_z, double rtol, int max_vcycles, void* stream, vdi_mg_result* res) {
    using namespace vdi;
    if (!d_b || !d_z || !(rtol > 0) || max_vcycles < 0 || kind < 0 || kind > 3 || m < 2 || n < 2) {
        set_error("vdi_mg_solve_noalloc: invalid arguments");
        return VDI_ERR_INVALID_ARGUMENT;
    }
    if (long(m) * n > NOALLOC_MAX_UNKNOWNS) {
        set_error("vdi_mg_solve_noalloc: %dx%d = %ld unknowns exceeds the maximum of %ld", m, n, long(m) * n,
                  NOALLOC_MAX_UNKNOWNS);
        return VDI_ERR_UNSUPPORTED_SIZE;
    }
    std::lock_guard<std::mutex> lock(noalloc_mutex());
    int dev = 0;
    VDI_CUDA(cudaGetDevice(&dev));
    unsigned char* base = nullptr;
    VDI_TRY(noalloc_base(dev, &base));
    NoallocKey key{dev, kind, m, n, x_sym, c1, c2};
    if (kind == VDI_MG_MAC) {
        // mgs_mac.cc:23-27 (test constructor): xxsp = 1/(dx*dx)
        key.c1 = 1. / (c1 * c1);
        key.c2 = 1. / (c2 * c2);
    }
    auto& cache = noalloc_cache();
    MG* g = nullptr;
    for (size_t q = 0; q < cache.size(); q++) {
        if (cache[q].key == key) {
            NoallocEntry hit = cache[q];      // most recently used goes last
            cache.erase(cache.begin() + q);
            cache.push_back(hit);
            g = hit.mg;
            break;
        }
    }
    if (!g) {
        VDI_TRY(noalloc_build(key, base, &g));
        if (cache.size() >= NOALLOC_CACHE_MAX) {
            noalloc_drop(cache.front().mg);
            cache.erase(cache.begin());
        }
        cache.push_back(NoallocEntry{key, g});
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the array keeps the previous call's contents: restart the control
    // block and the reduction counter
    VDI_CUDA(cudaMemsetAsync(g->ctl, 0, sizeof(SolveCtl), s));
    VDI_CUDA(cudaMemsetAsync(g->rd.counter, 0, sizeof(unsigned), s));
    VDI_TRY(g->set_ctl_params(s, rtol, max_vcycles));
    int v = 0;
    double r = 0;
    int st = mg_solve(g, s, d_b, d_z, rtol, max_vcycles, VDI_MG_FP64, &v, &r);
    if (res) {
        res->vcycles = v;
        res->rel_res = r;
    }
    return st;
}
