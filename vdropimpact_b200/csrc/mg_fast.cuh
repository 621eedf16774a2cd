// Separable exact coarse solve (included by mg.cu).
//
// The MAC operator (cell-centred, 5-point) is a Kronecker sum A = Ax (x) I +
// I (x) Ay, and the FEM operator (node-centred bilinear, 9-point) is
// Kx (x) My + Mx (x) Ky; both have natural (Neumann) ends in x. A cosine
// basis diagonalises their x parts: DCT-II for cells, DCT-I with half weights
// at the two end nodes for nodes (W = diag(1/2, 1, ..., 1, 1/2)). Writing
// each row of the source as b(., j) = W B beta(j) (B the basis, one mode per
// column), the system splits into one tridiagonal system in y per mode k:
//
//     tau_{k,-1}(j) a_k(j-1) + tau_{k,0}(j) a_k(j) + tau_{k,+1}(j) a_k(j+1) = beta_k(j)
//
// with beta(j) = C^-1 B^T b(., j), C = B^T W B (diagonal), and z(., j) = B a(j).
// The level is solved exactly in three launches: the forward transform (the
// rows times the scaled basis, a tiled product), the per-mode tridiagonal
// solves (parallel cyclic reduction in shared memory), and the inverse
// transform. A bottom row that holds only a
// diagonal (the FEM's Dirichlet nodes) is solved directly and its coupling
// into the next row moves to that row's source.
//
// Nothing is assumed about the operator beyond its 3 x 3 stencil: at setup
// the level's stencil is probed, the rows are grouped into classes of equal
// stencils, and for each class the basis is checked to diagonalise the
// class's three x operators to 1e-12; then a solve of a random source is
// checked against the operator. Any failure leaves the other coarse paths in
// place.

static constexpr int FC_T = 16;        // transform tile: 16 x 16 outputs, one per thread
static constexpr int FC_K = 64;        // transform chunk depth
static constexpr int FC_THREADS = 256;
static constexpr int FC_MAXROWS = 1024;   // rows of one mode's system (one thread each)

/** C[r][c] = sum_t A(r, t) B[t][c] over a row-major m x m matrix B, for
 * rows r < n - j0 and columns c < m; 16 x 16 tiles, one output per thread,
 * the next 64-deep chunk of A and B loaded into registers while the current
 * one is summed from shared memory.
 * FWD: A(r, t) = b(t, j0 + r) (the level's source, with the coupling of row
 * 1 to a directly solved Dirichlet row 0 subtracted when j0 = 1), C the
 * modal source beta at rows j0.. of out. Inverse: A(r, t) = in[(j0 + r) m +
 * t] (the modal solution), C the level's iterate; a Dirichlet row 0 is
 * z = b / dd. */
template <typename T, bool FWD>
__global__ void __launch_bounds__(FC_THREADS) fc_transform_k(const T* __restrict__ in, int m, int n, int j0,
                                                            const T* __restrict__ B, const T* __restrict__ b,
                                                            const T* __restrict__ dd, const T* __restrict__ dc,
                                                            T* __restrict__ out) {
    __shared__ T As[FC_K][FC_T + 1];   // [t][r]
    __shared__ T Bt[FC_K][FC_T + 1];   // [t][c]
    const int tid = threadIdx.x, tx = tid & (FC_T - 1), ty = tid / FC_T;
    const int r0 = blockIdx.y * FC_T, c0 = blockIdx.x * FC_T, rows = n - j0;
    if (!FWD && j0 == 1 && blockIdx.x == 0 && blockIdx.y == 0)
        for (int i = tid; i < m; i += blockDim.x) out[i] = b[i] / dd[i];
    auto a_at = [&](int r, int t) -> T {
        if (r >= rows || t >= m) return T(0);
        const int j = j0 + r;
        if (!FWD) return in[size_t(j) * m + t];
        T v = in[t + size_t(m) * j];
        if (j0 == 1 && j == 1) {
            T c = dc[m + t] * (in[t] / dd[t]);
            if (t > 0) c += dc[t] * (in[t - 1] / dd[t - 1]);
            if (t < m - 1) c += dc[2 * m + t] * (in[t + 1] / dd[t + 1]);
            v -= c;
        }
        return v;
    };
    auto b_at = [&](int t, int c) -> T { return (t < m && c < m) ? B[size_t(t) * m + c] : T(0); };
    constexpr int PER = FC_K * FC_T / FC_THREADS;   // 4 values of each tile per thread
    T pa[PER], pb[PER];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int e = tid + FC_THREADS * q;
            pa[q] = a_at(r0 + e / FC_K, k0 + e % FC_K);
            pb[q] = b_at(k0 + e / FC_T, c0 + e % FC_T);
        }
    };
    T acc = 0;
    fetch(0);
    for (int k0 = 0; k0 < m; k0 += FC_K) {
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int e = tid + FC_THREADS * q;
            As[e % FC_K][e / FC_K] = pa[q];
            Bt[e / FC_T][e % FC_T] = pb[q];
        }
        __syncthreads();
        if (k0 + FC_K < m) fetch(k0 + FC_K);
#pragma unroll 16
        for (int t = 0; t < FC_K; t++) acc += As[t][ty] * Bt[t][tx];
        __syncthreads();
    }
    const int r = r0 + ty, c = c0 + tx;
    if (r < rows && c < m) out[size_t(j0 + r) * m + c] = acc;
}

/** The per-mode tridiagonal systems over rows j0..n-1 of x[j][k] (source in,
 * solution out) by parallel cyclic reduction in shared memory: one thread
 * per row (rows padded to rp, a multiple of 32, with identity rows), mpb
 * modes per block. The reduction's coefficients do not depend on the source,
 * so they are precomputed: at step q (stride 2^q) row i's source becomes
 * d + AL[q] d(i - 2^q) + GA[q] d(i + 2^q), and at the end x = d IB. Layout
 * [q][i][k] (i the padded row) and [i][k]. */
template <typename T>
__global__ void __launch_bounds__(1024) fc_pcr_k(T* __restrict__ x, int m, int n, int j0, int rp, int mpb,
                                                 int steps, const T* __restrict__ AL, const T* __restrict__ GA,
                                                 const T* __restrict__ IB) {
    extern __shared__ __align__(16) unsigned char fc_raw[];
    T* sd = reinterpret_cast<T*>(fc_raw);
    const int g = threadIdx.x / rp, i = threadIdx.x - g * rp, k = blockIdx.x * mpb + g, R = n - j0;
    const int o = g * rp;
    const bool mode = k < m, real = mode && i < R;
    constexpr int QMAX = 10;   // rp <= 1024
    T al[QMAX], ga[QMAX];
    T d = 0, ib = 1;
    if (mode) {
        const size_t plane = size_t(rp) * m, q0 = size_t(i) * m + k;
#pragma unroll
        for (int q = 0; q < QMAX; q++)
            if (q < steps) {
                al[q] = AL[q * plane + q0];
                ga[q] = GA[q * plane + q0];
            }
        ib = IB[q0];
        if (real) d = x[size_t(j0 + i) * m + k];
    }
    sd[o + i] = d;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < QMAX; q++) {
        if (q >= steps) break;
        const int s = 1 << q;
        T dn = d;
        if (mode) {
            if (i - s >= 0) dn += al[q] * sd[o + i - s];
            if (i + s < rp) dn += ga[q] * sd[o + i + s];
        }
        __syncthreads();
        d = dn;
        sd[o + i] = d;
        __syncthreads();
    }
    if (real) x[size_t(j0 + i) * m + k] = d * ib;
}

/** Device arrays of the separable solve of one level, in one precision. */
template <typename T>
struct FastArrays {
    T *Bs = nullptr, *BT = nullptr;              // m x m: scaled basis, transposed basis
    T *AL = nullptr, *GA = nullptr, *IB = nullptr;   // cyclic reduction's coefficients
    T *dd = nullptr, *dc = nullptr;              // Dirichlet row: diagonal (m), coupling of row 1 (3 m)
    T* work = nullptr;                           // n x m
    void release() {
        for (T* p : {Bs, BT, AL, GA, IB, dd, dc, work})
            if (p) cudaFree(p);
        Bs = BT = AL = GA = IB = dd = dc = work = nullptr;
    }
};

/** Host analysis of a level's probed stencil (nine planes, plane
 * (dx+1) + 3 (dy+1), value at point i + m j). node: DCT-I with half end
 * weights (node-centred), else DCT-II. On success fills the basis, the
 * per-mode tridiagonal coefficients and the Dirichlet-row data in FP64 and
 * returns true. */
struct FastHost {
    int m = 0, n = 0, j0 = 0, rp = 0, steps = 0;
    std::vector<double> Bs, BT, AL, GA, IB, dd, dc;
};

static bool fast_analyse(const std::vector<double>& S, int m, int n, bool node, FastHost& F) {
    const long N = long(m) * n;
    auto s = [&](int dx, int dy, int i, int j) { return S[size_t((dx + 1) + 3 * (dy + 1)) * N + i + size_t(m) * j]; };
    if (m < 4 || n < 3) return false;
    double scale = 0;
    for (double v : S) scale = std::max(scale, std::fabs(v));
    if (!(scale > 0) || !std::isfinite(scale)) return false;
    // a bottom row holding only its diagonal is solved directly
    int j0 = 1;
    for (int i = 0; i < m && j0; i++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++)
                if ((dx || dy) && s(dx, dy, i, 0) != 0) j0 = 0;
    if (j0)
        for (int i = 0; i < m; i++)
            if (!(std::fabs(s(0, 0, i, 0)) > 1e-300)) return false;
    // the basis and its weights
    std::vector<double> B(size_t(m) * m), W(m, 1.0), C(m, 0.0);
    const double PI = 3.14159265358979323846;
    for (int i = 0; i < m; i++)
        for (int k = 0; k < m; k++)
            B[size_t(i) * m + k] = node ? std::cos(PI * k * i / (m - 1)) : std::cos(PI * k * (i + 0.5) / m);
    if (node) W[0] = W[m - 1] = 0.5;
    for (int k = 0; k < m; k++)
        for (int i = 0; i < m; i++) C[k] += B[size_t(i) * m + k] * W[i] * B[size_t(i) * m + k];
    // tau[dy+1][j][k], with rows grouped by equal stencils
    std::vector<double> tau(size_t(3) * n * m, 0.0);
    std::vector<int> rep(n, -1);
    std::vector<double> u(m);
    for (int j = j0; j < n; j++) {
        // an earlier row with the same stencil?
        for (int q = j0; q < j && rep[j] < 0; q++) {
            if (rep[q] != q) continue;
            bool same = true;
            for (int d = 0; d < 9 && same; d++)
                for (int i = 0; i < m && same; i++) same = S[size_t(d) * N + i + size_t(m) * j] == S[size_t(d) * N + i + size_t(m) * q];
            if (same) rep[j] = q;
        }
        if (rep[j] >= 0) {
            for (int d = 0; d < 3; d++)
                for (int k = 0; k < m; k++) tau[(size_t(d) * n + j) * m + k] = tau[(size_t(d) * n + rep[j]) * m + k];
            continue;
        }
        rep[j] = j;
        for (int dy = -1; dy <= 1; dy++) {
            for (int k = 0; k < m; k++) {
                // u = R v_k, R the x operator coupling row j to row j+dy
                double num = 0, err = 0;
                for (int i = 0; i < m; i++) {
                    double v = 0;
                    for (int dx = -1; dx <= 1; dx++) {
                        const int ii = i + dx;
                        if (ii < 0 || ii >= m) continue;
                        v += s(dx, dy, i, j) * B[size_t(ii) * m + k];
                    }
                    u[i] = v;
                    num += B[size_t(i) * m + k] * v;
                }
                const double t = num / C[k];
                for (int i = 0; i < m; i++) err = std::max(err, std::fabs(u[i] - t * W[i] * B[size_t(i) * m + k]));
                if (!(err <= 1e-12 * scale)) return false;
                tau[(size_t(dy + 1) * n + j) * m + k] = t;
            }
        }
    }
    // the tridiagonal systems per mode over rows j0..n-1 (the coupling of row
    // j0 to a Dirichlet row below moves to the source); elimination without
    // pivoting must not meet a vanishing pivot
    const int R = n - j0;
    if (R > FC_MAXROWS) return false;
    const int rp = (R + 31) / 32 * 32;
    int steps = 0;
    while ((1 << steps) < rp) steps++;
    F.AL.assign(size_t(steps) * rp * m, 0.0);
    F.GA.assign(size_t(steps) * rp * m, 0.0);
    F.IB.assign(size_t(rp) * m, 1.0);
    std::vector<double> a(rp), bb(rp), c(rp), a2(rp), b2(rp), c2(rp);
    for (int k = 0; k < m; k++) {
        double cprev = 0;
        for (int i = 0; i < rp; i++) {
            const int j = j0 + i;
            if (i < R) {
                a[i] = i > 0 ? tau[(size_t(0) * n + j) * m + k] : 0.0;
                bb[i] = tau[(size_t(1) * n + j) * m + k];
                c[i] = i < R - 1 ? tau[(size_t(2) * n + j) * m + k] : 0.0;
                const double den = bb[i] - a[i] * cprev;
                if (!(std::fabs(den) > 1e-13 * scale)) return false;
                cprev = c[i] / den;
            } else {
                a[i] = 0;
                bb[i] = 1;
                c[i] = 0;
            }
        }
        // cyclic reduction of the coefficients (the source is reduced on the
        // device with the same factors)
        for (int q = 0; q < steps; q++) {
            const int st = 1 << q;
            for (int i = 0; i < rp; i++) {
                const double al = i - st >= 0 ? -a[i] / bb[i - st] : 0.0;
                const double ga = i + st < rp ? -c[i] / bb[i + st] : 0.0;
                F.AL[(size_t(q) * rp + i) * m + k] = al;
                F.GA[(size_t(q) * rp + i) * m + k] = ga;
                a2[i] = i - st >= 0 ? al * a[i - st] : 0.0;
                c2[i] = i + st < rp ? ga * c[i + st] : 0.0;
                b2[i] = bb[i] + (i - st >= 0 ? al * c[i - st] : 0.0) + (i + st < rp ? ga * a[i + st] : 0.0);
            }
            a.swap(a2);
            bb.swap(b2);
            c.swap(c2);
        }
        for (int i = 0; i < rp; i++) {
            if (!(std::fabs(bb[i]) > 1e-300)) return false;
            F.IB[size_t(i) * m + k] = 1.0 / bb[i];
        }
    }
    F.rp = rp;
    F.steps = steps;
    F.m = m;
    F.n = n;
    F.j0 = j0;
    F.Bs.resize(size_t(m) * m);
    F.BT.resize(size_t(m) * m);
    for (int i = 0; i < m; i++)
        for (int k = 0; k < m; k++) {
            F.Bs[size_t(i) * m + k] = B[size_t(i) * m + k] / C[k];
            F.BT[size_t(k) * m + i] = B[size_t(i) * m + k];
        }
    F.dd.assign(m, 1.0);
    F.dc.assign(size_t(3) * m, 0.0);
    if (j0) {
        for (int i = 0; i < m; i++) {
            F.dd[i] = s(0, 0, i, 0);
            for (int dx = -1; dx <= 1; dx++) F.dc[size_t(dx + 1) * m + i] = s(dx, -1, i, 1);
        }
    }
    return true;
}

/** Uploads the analysis in precision T. */
template <typename T>
static int fast_upload(const FastHost& F, FastArrays<T>& A) {
    auto up = [](const std::vector<double>& h, T** d) -> int {
        std::vector<T> t(h.begin(), h.end());
        VDI_CUDA(cudaMalloc(d, t.size() * sizeof(T)));
        VDI_CUDA(cudaMemcpy(*d, t.data(), t.size() * sizeof(T), cudaMemcpyHostToDevice));
        return VDI_OK;
    };
    VDI_TRY(up(F.Bs, &A.Bs));
    VDI_TRY(up(F.BT, &A.BT));
    VDI_TRY(up(F.AL, &A.AL));
    VDI_TRY(up(F.GA, &A.GA));
    VDI_TRY(up(F.IB, &A.IB));
    VDI_TRY(up(F.dd, &A.dd));
    VDI_TRY(up(F.dc, &A.dc));
    VDI_CUDA(cudaMalloc(&A.work, size_t(F.n) * F.m * sizeof(T)));
    return VDI_OK;
}

/** The exact solve z = A^-1 b of the level on stream s (rp, steps: the
 * padded rows and the reduction steps of the analysis). */
template <typename T>
static int fast_solve(cudaStream_t s, const FastArrays<T>& A, int m, int n, int j0, int rp, int steps, const T* b,
                      T* z) {
    const dim3 grid((m + FC_T - 1) / FC_T, (n - j0 + FC_T - 1) / FC_T);
    fc_transform_k<T, true><<<grid, FC_THREADS, 0, s>>>(b, m, n, j0, A.Bs, b, A.dd, A.dc, A.work);
    const int mpb = std::max(1, 512 / rp);
    fc_pcr_k<T><<<(m + mpb - 1) / mpb, rp * mpb, size_t(rp) * mpb * sizeof(T), s>>>(A.work, m, n, j0, rp, mpb, steps,
                                                                                   A.AL, A.GA, A.IB);
    fc_transform_k<T, false><<<grid, FC_THREADS, 0, s>>>(A.work, m, n, j0, A.BT, b, A.dd, A.dc, z);
    VDI_CUDA(cudaGetLastError());
    return VDI_OK;
}
