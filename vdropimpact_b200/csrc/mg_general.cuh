// Multigrid for grids of any size (included by mg.cu).
//
// The constant-stencil hierarchy of mg.cu halves cell grids while both sides
// are even and node grids while both interval counts are even; other sizes
// (an odd factor left in a side, as in the reference's mg_test sizes or a
// 5120x960 run) stop it at a level too large for its coarsest smoother. For
// those the solver switches to this path:
//   - level 0 is the problem's own operator, assembled into a stored 9-point
//     stencil by applying it to nine lattice probes (one unknown in every 3x3
//     block), so it is the operator of the fast path exactly;
//   - vertex-style coarsening of each side longer than two points (coarse
//     point I on fine point 2I; an odd-indexed last fine point takes the last
//     coarse value), bilinear prolongation P, restriction P^T and Galerkin
//     coarse operators P^T A P, again 9-point stencils;
//   - four-colour Gauss-Seidel (the ordering that is a true Gauss-Seidel for
//     9-point stencils), two sweeps before and after the coarse correction;
//   - the coarsest level (at most GEN_MAX_COARSE unknowns) solved with its
//     inverse, formed once on the host by Gauss-Jordan elimination with
//     partial pivoting.
// Stencils are stored as nine planes S[d][ij], d = 3 (dy+1) + (dx+1).

static constexpr int GEN_MAX_COARSE = 512;

struct GenOp {
    const double* S;
    int m, n;
};

__device__ __forceinline__ int op_m(const GenOp& c) { return c.m; }
__device__ __forceinline__ int op_n(const GenOp& c) { return c.n; }

/** b - A z at (i,j), w = z + i + P j. */
template <typename T>
__device__ __forceinline__ T op_resid(const GenOp& c, const T* w, T bv, int P, int i, int j) {
    const long mn = long(c.m) * c.n, k = i + long(P) * j;
    double acc = double(bv);
#pragma unroll
    for (int dy = -1; dy <= 1; dy++) {
        if (j + dy < 0 || j + dy >= c.n) continue;
#pragma unroll
        for (int dx = -1; dx <= 1; dx++) {
            if (i + dx < 0 || i + dx >= c.m) continue;
            acc -= c.S[(3 * (dy + 1) + dx + 1) * mn + k] * double(w[dx + long(P) * dy]);
        }
    }
    return T(acc);
}

/** Lattice probe: 1 where i%3 == px and j%3 == py. */
__global__ void gen_probe_k(double* p, int m, int n, int px, int py) {
    long tot = long(m) * n;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < tot; k += long(gridDim.x) * blockDim.x) {
        int j = int(k / m), i = int(k - long(j) * m);
        p[k] = (i % 3 == px && j % 3 == py) ? 1. : 0.;
    }
}

/** y = A p for a lattice probe holds, at each point, its coupling to the one
 * probe point in its 3x3 neighbourhood. */
__global__ void gen_extract_k(const double* y, double* S, int m, int n, int px, int py) {
    long tot = long(m) * n;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < tot; k += long(gridDim.x) * blockDim.x) {
        int j = int(k / m), i = int(k - long(j) * m);
        int ex = ((px - i) % 3 + 3) % 3, ey = ((py - j) % 3 + 3) % 3;
        int dx = ex == 2 ? -1 : ex, dy = ey == 2 ? -1 : ey;
        S[(3 * (dy + 1) + dx + 1) * tot + k] = y[k];
    }
}

/** The 1-D prolongation weights: the coarse points (at most two) whose
 * basis functions cover fine point i, and their weights. */
__device__ __forceinline__ int gen_p1(int i, int mf, int mc, int* I, double* w) {
    if (mc == mf) {             // this side is not coarsened
        I[0] = i;
        w[0] = 1.;
        return 1;
    }
    if (!(i & 1)) {
        I[0] = i >> 1;
        w[0] = 1.;
        return 1;
    }
    int a = (i - 1) >> 1, b = (i + 1) >> 1;
    if (b >= mc) {              // last fine point past the last coarse point
        I[0] = a;
        w[0] = 1.;
        return 1;
    }
    I[0] = a;
    w[0] = 0.5;
    I[1] = b;
    w[1] = 0.5;
    return 2;
}

/** The fine points covered by coarse point I's basis function: [lo, hi]. */
__device__ __forceinline__ void gen_support(int I, int mf, int mc, int* lo, int* hi) {
    if (mc == mf) {
        *lo = *hi = I;
        return;
    }
    *lo = max(2 * I - 1, 0);
    *hi = min(2 * I + 1, mf - 1);
    if (I == mc - 1) *hi = mf - 1;
}

/** Galerkin coarse stencil A_c = P^T A P at each coarse point. */
__global__ void gen_rap_k(const double* __restrict__ Sf, int mf, int nf, double* __restrict__ Sc, int mc, int nc) {
    const long totc = long(mc) * nc, totf = long(mf) * nf;
    for (long K = blockIdx.x * long(blockDim.x) + threadIdx.x; K < totc; K += long(gridDim.x) * blockDim.x) {
        const int J = int(K / mc), I = int(K - long(J) * mc);
        double acc[9];
#pragma unroll
        for (int d = 0; d < 9; d++) acc[d] = 0.;
        int ilo, ihi, jlo, jhi;
        gen_support(I, mf, mc, &ilo, &ihi);
        gen_support(J, nf, nc, &jlo, &jhi);
        for (int j = jlo; j <= jhi; j++) {
            int Jy[2];
            double wy[2];
            int ny = gen_p1(j, nf, nc, Jy, wy);
            double pj = 0;
            for (int q = 0; q < ny; q++)
                if (Jy[q] == J) pj = wy[q];
            if (pj == 0) continue;
            for (int i = ilo; i <= ihi; i++) {
                int Ix[2];
                double wx[2];
                int nx = gen_p1(i, mf, mc, Ix, wx);
                double pi = 0;
                for (int q = 0; q < nx; q++)
                    if (Ix[q] == I) pi = wx[q];
                if (pi == 0) continue;
                const double pw = pi * pj;
                const long kf = i + long(mf) * j;
                for (int dy = -1; dy <= 1; dy++) {
                    const int l = j + dy;
                    if (l < 0 || l >= nf) continue;
                    int Ly[2];
                    double vy[2];
                    int nly = gen_p1(l, nf, nc, Ly, vy);
                    for (int dx = -1; dx <= 1; dx++) {
                        const int k = i + dx;
                        if (k < 0 || k >= mf) continue;
                        const double a = Sf[(3 * (dy + 1) + dx + 1) * totf + kf];
                        if (a == 0) continue;
                        int Lx[2];
                        double vx[2];
                        int nlx = gen_p1(k, mf, mc, Lx, vx);
                        for (int qy = 0; qy < nly; qy++)
                            for (int qx = 0; qx < nlx; qx++) {
                                const int ex = Lx[qx] - I, ey = Ly[qy] - J;
                                acc[3 * (ey + 1) + ex + 1] += pw * a * vx[qx] * vy[qy];
                            }
                    }
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 9; d++) Sc[d * totc + K] = acc[d];
    }
}

/** One colour of four-colour Gauss-Seidel (colour = (i&1) + 2 (j&1)). */
__global__ void gen_smooth_k(GenOp c, double* __restrict__ z, const double* __restrict__ b, int color) {
    const int mh = (c.m + 1 - (color & 1)) >> 1, nh = (c.n + 1 - (color >> 1)) >> 1;
    const long tot = long(mh) * nh, mn = long(c.m) * c.n;
    for (long q = blockIdx.x * long(blockDim.x) + threadIdx.x; q < tot; q += long(gridDim.x) * blockDim.x) {
        const int jh = int(q / mh), ih = int(q - long(jh) * mh);
        const int i = 2 * ih + (color & 1), j = 2 * jh + (color >> 1);
        const long k = i + long(c.m) * j;
        double r = op_resid(c, z + k, b[k], c.m, i, j);
        z[k] += r / c.S[4 * mn + k];
    }
}

/** b_c = P^T (b - A z) at each coarse point (the fine residual recomputed at
 * the points of the basis function's support). */
__global__ void gen_restrict_k(GenOp f, const double* __restrict__ z, const double* __restrict__ b,
                               double* __restrict__ bc, int mc, int nc) {
    const long totc = long(mc) * nc;
    for (long K = blockIdx.x * long(blockDim.x) + threadIdx.x; K < totc; K += long(gridDim.x) * blockDim.x) {
        const int J = int(K / mc), I = int(K - long(J) * mc);
        int ilo, ihi, jlo, jhi;
        gen_support(I, f.m, mc, &ilo, &ihi);
        gen_support(J, f.n, nc, &jlo, &jhi);
        double acc = 0;
        for (int j = jlo; j <= jhi; j++) {
            int Jy[2];
            double wy[2];
            int ny = gen_p1(j, f.n, nc, Jy, wy);
            double pj = 0;
            for (int q = 0; q < ny; q++)
                if (Jy[q] == J) pj = wy[q];
            if (pj == 0) continue;
            for (int i = ilo; i <= ihi; i++) {
                int Ix[2];
                double wx[2];
                int nx = gen_p1(i, f.m, mc, Ix, wx);
                double pi = 0;
                for (int q = 0; q < nx; q++)
                    if (Ix[q] == I) pi = wx[q];
                if (pi == 0) continue;
                const long k = i + long(f.m) * j;
                acc += pi * pj * op_resid(f, z + k, b[k], f.m, i, j);
            }
        }
        bc[K] = acc;
    }
}

/** z += P z_c. */
__global__ void gen_prolong_k(double* __restrict__ z, int mf, int nf, const double* __restrict__ zc, int mc, int nc) {
    const long tot = long(mf) * nf;
    for (long k = blockIdx.x * long(blockDim.x) + threadIdx.x; k < tot; k += long(gridDim.x) * blockDim.x) {
        const int j = int(k / mf), i = int(k - long(j) * mf);
        int Ix[2], Jy[2];
        double wx[2], wy[2];
        int nx = gen_p1(i, mf, mc, Ix, wx), ny = gen_p1(j, nf, nc, Jy, wy);
        double v = 0;
        for (int qy = 0; qy < ny; qy++)
            for (int qx = 0; qx < nx; qx++) v += wx[qx] * wy[qy] * zc[Ix[qx] + long(mc) * Jy[qy]];
        z[k] += v;
    }
}

/** z = Ainv b on the coarsest level (one thread per row). */
__global__ void gen_coarse_k(const double* __restrict__ inv, const double* __restrict__ b, double* __restrict__ z,
                             int N) {
    extern __shared__ double sb[];
    for (int k = threadIdx.x; k < N; k += blockDim.x) sb[k] = b[k];
    __syncthreads();
    for (int r = threadIdx.x; r < N; r += blockDim.x) {
        double s = 0;
        const double* row = inv + long(r) * N;
        for (int k = 0; k < N; k++) s += row[k] * sb[k];
        z[r] = s;
    }
}

/** The inverse (row-major, N = m n) of the operator given by nine stencil
 * planes on the device, formed on the host by Gauss-Jordan elimination with
 * partial pivoting; for the small coarsest levels only. */
static int stencil_inverse(const double* d_S, int m, int n, std::vector<double>& X, bool pin_mean = false) {
    const int N = m * n;
    std::vector<double> Sc(9 * size_t(N));
    VDI_CUDA(cudaMemcpy(Sc.data(), d_S, Sc.size() * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<double> A(size_t(N) * N, 0.);
    X.assign(size_t(N) * N, 0.);
    for (int k = 0; k < N; k++) {
        int j = k / m, i = k - j * m;
        for (int d = 0; d < 9; d++) {
            int dx = d % 3 - 1, dy = d / 3 - 1;
            int ii = i + dx, jj = j + dy;
            if (ii < 0 || ii >= m || jj < 0 || jj >= n) continue;
            A[size_t(k) * N + ii + size_t(m) * jj] += Sc[size_t(d) * N + k];
        }
        X[size_t(k) * N + k] = 1.;
    }
    if (pin_mean) {
        // a singular Neumann operator (constants in its null space): the last
        // equation, redundant for a consistent source, becomes "sum = 0"
        for (int q = 0; q < N; q++) A[size_t(N - 1) * N + q] = 1.;
    }
    for (int c = 0; c < N; c++) {
        int piv = c;
        for (int r = c + 1; r < N; r++)
            if (std::fabs(A[size_t(r) * N + c]) > std::fabs(A[size_t(piv) * N + c])) piv = r;
        if (A[size_t(piv) * N + c] == 0) {
            set_error("multigrid: singular coarsest operator (%d unknowns)", N);
            return VDI_ERR_UNSUPPORTED_SIZE;
        }
        if (piv != c)
            for (int q = 0; q < N; q++) {
                std::swap(A[size_t(c) * N + q], A[size_t(piv) * N + q]);
                std::swap(X[size_t(c) * N + q], X[size_t(piv) * N + q]);
            }
        const double d = 1. / A[size_t(c) * N + c];
        for (int q = 0; q < N; q++) {
            A[size_t(c) * N + q] *= d;
            X[size_t(c) * N + q] *= d;
        }
        for (int r = 0; r < N; r++) {
            if (r == c) continue;
            const double f = A[size_t(r) * N + c];
            if (f == 0) continue;
            for (int q = 0; q < N; q++) {
                A[size_t(r) * N + q] -= f * A[size_t(c) * N + q];
                X[size_t(r) * N + q] -= f * X[size_t(c) * N + q];
            }
        }
    }
    if (pin_mean)
        for (int r = 0; r < N; r++) X[size_t(r) * N + N - 1] = 0.;   // the constraint's right-hand side is 0
    return VDI_OK;
}

/** Nine stencil planes of an operator on an m x n grid, probed through
 * apply(p, y) (y = A p) with the nine lattice vectors. */
template <class APPLY>
static int probe_stencil(int m, int n, double* d_S, APPLY apply) {
    const long N = long(m) * n;
    double *p, *y;
    VDI_CUDA(cudaMalloc(&p, N * sizeof(double)));
    VDI_CUDA(cudaMalloc(&y, N * sizeof(double)));
    int st = VDI_OK;
    const int nb = std::max(1, std::min(nblk(N), 4096));
    for (int py = 0; py < 3 && st == VDI_OK; py++)
        for (int px = 0; px < 3 && st == VDI_OK; px++) {
            gen_probe_k<<<nb, 256>>>(p, m, n, px, py);
            st = apply(p, y);
            if (st == VDI_OK) gen_extract_k<<<nb, 256>>>(y, d_S, m, n, px, py);
        }
    cudaError_t e = cudaDeviceSynchronize();
    cudaFree(p);
    cudaFree(y);
    VDI_TRY(st);
    VDI_CUDA(e);
    return VDI_OK;
}

/** The general hierarchy of one system. */
struct GenMG {
    std::vector<int> gm, gn;          // level sizes
    std::vector<double*> S;           // stencils, 9 planes per level
    std::vector<double*> z, b;        // level iterates and sources (level 0: the caller's)
    double* inv = nullptr;            // coarsest inverse
    int N = 0;                        // coarsest unknowns

    int nlev() const { return int(gm.size()); }
    long size(int l) const { return long(gm[l]) * gn[l]; }
    GenOp op(int l) const { return GenOp{S[l], gm[l], gn[l]}; }

    void release() {
        for (auto p : S) if (p) cudaFree(p);
        for (auto p : z) if (p) cudaFree(p);
        for (auto p : b) if (p) cudaFree(p);
        if (inv) cudaFree(inv);
        S.clear(); z.clear(); b.clear();
        inv = nullptr;
        gm.clear(); gn.clear();
    }

    /** Builds the hierarchy; apply(z, y) computes y = A z on level 0. */
    template <class APPLY>
    int setup(int m, int n, APPLY apply, bool pin_mean = false) {
        release();
        gm.push_back(m);
        gn.push_back(n);
        while (long(gm.back()) * gn.back() > GEN_MAX_COARSE && int(gm.size()) < 24) {
            int mm = gm.back(), nn = gn.back();
            int mc = mm > 2 ? (mm + 1) / 2 : mm, nc = nn > 2 ? (nn + 1) / 2 : nn;
            if (mc == mm && nc == nn) break;
            gm.push_back(mc);
            gn.push_back(nc);
        }
        N = int(size(nlev() - 1));
        if (N > 4096) {
            set_error("multigrid: %dx%d grid does not coarsen below %d unknowns", m, n, N);
            return VDI_ERR_UNSUPPORTED_SIZE;
        }
        S.assign(nlev(), nullptr);
        z.assign(nlev(), nullptr);
        b.assign(nlev(), nullptr);
        for (int l = 0; l < nlev(); l++) {
            VDI_CUDA(cudaMalloc(&S[l], 9 * size(l) * sizeof(double)));
            if (l > 0) {
                VDI_CUDA(cudaMalloc(&z[l], size(l) * sizeof(double)));
                VDI_CUDA(cudaMalloc(&b[l], size(l) * sizeof(double)));
            }
        }
        // level 0: nine probes of the operator
        VDI_TRY(probe_stencil(m, n, S[0], apply));
        for (int l = 1; l < nlev(); l++)
            gen_rap_k<<<std::min(nblk(size(l)), 4096), 256>>>(S[l - 1], gm[l - 1], gn[l - 1], S[l], gm[l], gn[l]);
        VDI_CUDA(cudaGetLastError());
        // coarsest inverse by Gauss-Jordan with partial pivoting
        std::vector<double> X;
        VDI_TRY(stencil_inverse(S[nlev() - 1], gm[nlev() - 1], gn[nlev() - 1], X, pin_mean));
        VDI_CUDA(cudaMalloc(&inv, X.size() * sizeof(double)));
        VDI_CUDA(cudaMemcpy(inv, X.data(), X.size() * sizeof(double), cudaMemcpyHostToDevice));
        return VDI_OK;
    }

    int smooth(cudaStream_t s, int l, double* zl, const double* bl, bool reverse) {
        const int nb = std::max(1, std::min(nblk(size(l) / 4 + 1), 2048));
        for (int q = 0; q < 4; q++) gen_smooth_k<<<nb, 256, 0, s>>>(op(l), zl, bl, reverse ? 3 - q : q);
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    /** One V-cycle from level l on (bl, zl). */
    int vcycle(cudaStream_t s, int l, const double* bl, double* zl) {
        if (l == nlev() - 1) {
            gen_coarse_k<<<1, 1024, N * sizeof(double), s>>>(inv, bl, zl, N);
            VDI_CUDA(cudaGetLastError());
            return VDI_OK;
        }
        for (int k = 0; k < 2; k++) VDI_TRY(smooth(s, l, zl, bl, false));
        gen_restrict_k<<<std::max(1, std::min(nblk(size(l + 1)), 4096)), 256, 0, s>>>(op(l), zl, bl, b[l + 1],
                                                                                      gm[l + 1], gn[l + 1]);
        VDI_CUDA(cudaMemsetAsync(z[l + 1], 0, size(l + 1) * sizeof(double), s));
        VDI_TRY(vcycle(s, l + 1, b[l + 1], z[l + 1]));
        gen_prolong_k<<<std::max(1, std::min(nblk(size(l)), 4096)), 256, 0, s>>>(zl, gm[l], gn[l], z[l + 1],
                                                                                gm[l + 1], gn[l + 1]);
        for (int k = 0; k < 2; k++) VDI_TRY(smooth(s, l, zl, bl, true));
        VDI_CUDA(cudaGetLastError());
        return VDI_OK;
    }

    /** Kernels (and memsets) one V-cycle launches. */
    int kernels_per_vcycle() const { return (nlev() - 1) * (16 + 3) + 1; }
};
