// Internal declarations shared by the CUDA translation units of libvdi.
#pragma once

#include <cuda_runtime.h>
#include <cstdio>
#include <cstdarg>
#include <vector>

#include "vdi.h"

namespace vdi {

/** Records a message retrievable through vdi_last_error(). */
void set_error(const char* fmt, ...);

#define VDI_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            vdi::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,               \
                           cudaGetErrorString(e_));                                 \
            return e_ == cudaErrorMemoryAllocation ? VDI_ERR_OUT_OF_MEMORY         \
                                                   : VDI_ERR_CUDA;                  \
        }                                                                           \
    } while (0)

#define VDI_TRY(expr)                  \
    do {                               \
        int s_ = (expr);               \
        if (s_ != VDI_OK) return s_;   \
    } while (0)

/** Bits of the device-side error word. */
enum DevErr : int {
    DEV_MG_NOT_CONVERGED = 1,
    DEV_NEWTON = 2,
    DEV_TRI_SINGULAR = 4,
    DEV_NONFINITE = 8,
    DEV_DUP_TIME = 16
};

/** Device-resident bookkeeping of one linear solve, read by the host in
 * eager mode and by the loop-control kernel inside CUDA graphs. */
struct SolveCtl {
    double bnorm2;      // ||b||^2
    double rnorm2;      // ||b - A z||^2 of the current iterate
    double rtol;
    int it;             // V-cycles taken in the current solve
    int max_it;
    int done;           // 1 once converged or failed
    int status;         // DevErr bits
    // totals since the last statistics reset
    long long solves;
    long long vcycles;
    double last_rel;
    int sticky;         // DevErr bits of every solve since creation
    int* err_out;       // when set, a failing solve also ORs its bits here
    int tma_timeout;    // set when a tile kernel's bulk copy did not arrive in time
};

/** Deterministic block-then-grid sum: each block writes one partial, the
 * last block to finish adds the partials in index order. */
struct Reduce {
    double* partials = nullptr;   // [max_blocks]
    unsigned* counter = nullptr;  // 1 word, returns to 0 after each use
    int max_blocks = 0;
};

int reduce_alloc(Reduce& r, int max_blocks);
void reduce_free(Reduce& r);

/** Cell-centred operator of the MAC projection (mgs_mac.hh:25-50) or the
 * implicit viscous system (visco_impl.hh:28-53) on one multigrid level. */
struct CCOp {
    int visc;           // 0: MAC, 1: viscous
    int m, n;
    double kx, ky;      // MAC: xxsp, yysp; viscous: vfx, vfy (scaled per level)
    int x_sym, horiz;
    // homogeneous ghost multipliers for cell-centred interpolation
    signed char gL, gR, gD, gU;
};

/** Node-centred bilinear finite-element operator (mgs_fem.hh:42-57). */
struct FEMOp {
    int M, N;
    double fm, fey, hey, fex, hex, fc;
};

class MG;

/** Creates a multigrid hierarchy. For MAC c1,c2 = xxsp,yysp (squared inverse
 * spacings); FEM c1,c2 = dx,dy;
 * viscous c1,c2 = vfx,vfy. */
int mg_create(int kind, int m, int n, double c1, double c2, int x_sym, MG** out);
void mg_destroy(MG* mg);
/** Re-derives the viscous coefficients (visco_impl::setup_and_solve
 * re-setup when vfx changes, visco_impl.cc:26-30). */
/** Bytes below which levels run in the single-CTA cycle (rebuilds). */
int mg_set_cta_limit(MG* mg, size_t bytes);
size_t mg_cta_limit(const MG* mg);
/** First level of the single-launch coarse cycle (-1: none) and the CTAs it
 * runs on (1: one CTA; more: a cluster). */
int mg_coarse_cycle(const MG* mg, int precision, int* first, int* ctas);
/** Tiled (per-launch) levels of the hierarchy for a precision; -1 for the
 * general hierarchy. */
int mg_tiled_levels(const MG* mg, int precision);
int mg_set_visc(MG* mg, double vfx, double vfy);
/** Solves A z = b on the stream. z holds the initial guess. Returns a
 * VDI_* status; eager mode reads the convergence state on the host. */
int mg_solve(MG* mg, cudaStream_t s, const double* b, double* z, double rtol, int max_it,
             int precision, int* vcycles, double* rel_res);
/** Enqueues a device-controlled solve (no host synchronisation): the loop
 * control lives in ctl and is driven by graph conditional nodes when
 * capturing, else unrolled up to max_unrolled V-cycles guarded by ctl. */
int mg_solve_device(MG* mg, cudaStream_t s, const double* b, double* z, int precision);
int mg_v_cycle(MG* mg, cudaStream_t s, const double* b, double* z);
int mg_residual(MG* mg, cudaStream_t s, const double* b, const double* z, double* r, double* norm);
int mg_apply(MG* mg, cudaStream_t s, const double* z, double* y);
SolveCtl* mg_ctl(MG* mg);          // device pointer
int mg_kind(const MG* mg);
int mg_fine_size(const MG* mg);    // number of unknowns on the finest level
int mg_dims(const MG* mg, int* m, int* n);   // finest level: cells (MAC, viscous) or nodes (FEM)
/** Configures the device-controlled solve (rtol, V-cycle cap). */
int mg_configure(MG* mg, double rtol, int max_it);
/** A device word that failing solves OR their DevErr bits into (the
 * owner's error word), kept across rebuilds of the hierarchy. */
int mg_set_error_word(MG* mg, int* d_err);
/* The finest-tile variant (0 shared memory, 1 and 2 register-blocked, 3
 * persistent TMA-fed for FP64 cell-centred levels) and the persistent
 * tile's launches so far. */
int mg_tile_path(long long* persistent_launches);
/** Builds the conditional-node loop for the solve into a graph under
 * stream capture. Returns VDI_OK when a graph loop was recorded. */
int mg_record_graph_solve(MG* mg, cudaStream_t s, const double* b, double* z, int precision);
/** Kernel launches of one solve-loop iteration (a V-cycle and its norm). */
int mg_kernels_per_iteration(const MG* mg, int precision);
/** Times the finest-level PRE (which=0) or POST (which=1) kernel. */
int mg_profile(MG* mg, cudaStream_t s, int which, int iters, const double* b, double* z, float* ms,
               double* bytes);

/** Canonical algorithmic bytes of one V-cycle: (3 (nu1 + nu2) + 4.5) words
 * per point of every level, the finest level's words fine_word bytes and the
 * coarser levels' coarse_word bytes. */
double mg_vcycle_bytes(const MG* mg, int fine_word, int coarse_word);

/** r = b - A z on the finest level and ||r||_2 into *d_norm, on the stream
 * without host synchronisation (graph-capturable). */
int mg_residual_async(MG* mg, cudaStream_t s, const double* b, const double* z, double* r, double* d_norm);

/** Learned correction of an initial guess: restricts r (m x n) by factor,
 * normalises by its RMS (from d_rnorm = ||r||_2), runs the U-Net and adds
 * scale * rms * (prolonged output) to z. in_buf/out_buf hold H x W floats. */
int unet_correct(vdi_unet* u, cudaStream_t s, const double* r, const double* d_rnorm, double* z, int m, int n,
                 int factor, double scale, float* in_buf, float* out_buf);
/** Kernels one unet_correct call launches. */
int unet_kernels_per_correction();
int unet_dims(const vdi_unet* u, int* H, int* W);

}  // namespace vdi
