// Cluster-resident coarse cycle (included by mg.cu).
//
// The coarse levels of a V-cycle, from the cluster's top level down to the
// level solved exactly with its inverse, run in ONE launch of a thread-block
// cluster of CS CTAs (8 or 16, one per SM). Each CTA owns a slab of rows of
// every level, plus G ghost rows on each side, in its shared memory:
//
//   rows lo-G .. hi+G-1 of z and b, lo = rank*h, hi = lo+h (h = n/CS)
//
// Smoothing works like the tile kernels, on a halo that shrinks by one row
// per colour phase: the four red-black phases of a pre- or post-smoothing
// cover rows [lo-4,hi+4), [lo-3,hi+3), [lo-2,hi+2), [lo-1,hi+1) and leave
// exact values on the rows they need, so consecutive phases need only
// __syncthreads. Rows cross between CTAs through distributed shared memory
// at two points per level, each followed by one cluster barrier:
//   down: the final pre-smoothed rows (for the other CTAs' later
//         prolongation) and the restricted source of the next level (the
//         next level's ghost rows);
//   up:   the final post-smoothed rows (the finer level's prolongation
//         reads the coarse correction three rows beyond a slab).
// The last distributed level's residual goes to every CTA, and each CTA
// solves the exact level for the rows its prolongation reads.
//
// Every value a CTA computes for a ghost row equals what the owning CTA
// computes for it, so the cycle does the same arithmetic as the single-CTA
// cycle and the tile kernels.
static constexpr int CL_MAXLEV = 8;
static constexpr int CL_THREADS = 512;
static constexpr int CL_G = 5;                       // ghost rows on each side (cell-centred)
static constexpr size_t CL_SMEM_LIMIT = 220 * 1024;  // per CTA

__device__ __forceinline__ void cl_arrive_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cl_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cl_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }
__device__ __forceinline__ int cl_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
    return int(r);
}
/** The same shared-memory location in CTA `rank` of the cluster. */
template <typename T>
__device__ __forceinline__ T* cl_map(T* p, int rank) {
    return cooperative_groups::this_cluster().map_shared_rank(p, unsigned(rank));
}

template <typename T>
struct CCClusterArgs {
    int nd;                    // distributed levels (lv[0] is the cluster's top level)
    int cs;                    // CTAs in the cluster
    CCc<T> lv[CL_MAXLEV];
    int h[CL_MAXLEV];          // own rows per CTA
    // shared-memory element offsets of each level's arrays:
    //   z, b: rows lo-G .. hi+G-1;  pre: final pre-smoothed rows lo-4..lo-1,
    //   hi..hi+3;  post: final post-smoothed rows lo-3..lo-1, hi..hi+2
    int oz[CL_MAXLEV], ob[CL_MAXLEV], opre[CL_MAXLEV], opost[CL_MAXLEV];
    CCc<T> dl;                 // the level solved exactly (the coarse level of lv[nd-1])
    const T* dinv;             // its inverse, row-major
    int ostage, odb, odz;      // residual of lv[nd-1] (all rows); source and solution of dl
};

/** Pushes row j of a slab level (src, m values) to every CTA that keeps it
 * as one of its D ghost rows on either side, into the array at element
 * offset `off` of that CTA: rows lo'-D..lo'-1 first, then hi'..hi'+D-1.
 * Called by one warp per row. */
template <typename T>
__device__ __forceinline__ void cl_push_row(T* sm, int off, const T* src, int m, int j, int r, int h, int cs,
                                            int D) {
    const int lane = threadIdx.x & 31;
    const int reach = (D + h - 1) / h;
    for (int d = -reach; d <= reach; d++) {
        const int t = r + d;
        if (d == 0 || t < 0 || t >= cs) continue;
        const int tlo = t * h, thi = tlo + h;
        int row;
        if (j < tlo && j >= tlo - D) row = j - (tlo - D);
        else if (j >= thi && j < thi + D) row = D + (j - thi);
        else continue;
        T* dst = cl_map(sm + off + row * m, t);
        for (int i = lane; i < m; i += 32) dst[i] = src[i];
    }
}

template <typename T>
__global__ void __launch_bounds__(CL_THREADS, 1) cc_cluster_cycle(CCClusterArgs<T> st, const T* __restrict__ gb,
                                                                   T* __restrict__ gz, int zero_init) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    constexpr int NW = CL_THREADS / 32, G = CL_G;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int r = cl_rank(), CS = st.cs;
    // no CTA touches another's shared memory before all have started
    cl_arrive_relaxed();
    auto zrow = [&](int q, int j) { return sm + st.oz[q] + (j - r * st.h[q] + G) * st.lv[q].m; };
    auto brow = [&](int q, int j) { return sm + st.ob[q] + (j - r * st.h[q] + G) * st.lv[q].m; };
    auto phase = [&](int q, int color, int a, int b) {
        const CCc<T>& c = st.lv[q];
        const int m = c.m;
        a = max(a, 0);
        b = min(b, c.n);
        for (int j = a + warp; j < b; j += NW) {
            T* zr = zrow(q, j);
            const T* br = brow(q, j);
            for (int i = 2 * lane + ((color ^ j) & 1); i < m; i += 64) zr[i] = op_relaxed(c, zr + i, br[i], m, i, j);
        }
        __syncthreads();
    };

    // the top level from global memory, with its ghost rows; coarser iterates start at zero
    {
        const CCc<T>& c = st.lv[0];
        const int m = c.m, lo = r * st.h[0], hi = lo + st.h[0];
        const int j0 = max(0, lo - G), j1 = min(c.n, hi + G);
        for (int j = j0 + warp; j < j1; j += NW) {
            T* zr = zrow(0, j);
            T* br = brow(0, j);
            for (int i = lane; i < m; i += 32) {
                br[i] = gb[i + size_t(m) * j];
                zr[i] = zero_init ? T(0) : gz[i + size_t(m) * j];
            }
        }
        for (int q = 1; q < st.nd; q++) {
            T* z = sm + st.oz[q];
            const int tot = (st.h[q] + 2 * G) * st.lv[q].m;
            for (int k = threadIdx.x; k < tot; k += CL_THREADS) z[k] = T(0);
        }
    }
    __syncthreads();

    // ---------------------------------------------------------------- down
    for (int q = 0; q < st.nd; q++) {
        const CCc<T>& c = st.lv[q];
        const int m = c.m, h = st.h[q], lo = r * h, hi = lo + h;
        phase(q, 0, lo - 4, hi + 4);
        phase(q, 1, lo - 3, hi + 3);
        phase(q, 0, lo - 2, hi + 2);
        phase(q, 1, lo - 1, hi + 1);
        if (q == 0) cl_wait();
        for (int j = lo + warp; j < hi; j += NW) cl_push_row(sm, st.opre[q], zrow(q, j), m, j, r, h, CS, 4);
        if (q + 1 < st.nd) {
            // restriction to the next level's own rows, and its ghost rows to the other CTAs
            const CCc<T>& cc = st.lv[q + 1];
            const int cm = cc.m, ch = st.h[q + 1], clo = r * ch, chi = clo + ch;
            const int reach = (4 + ch - 1) / ch;
            for (int J = clo + warp; J < chi; J += NW) {
                T* bd = brow(q + 1, J);
                for (int I = lane; I < cm; I += 32) {
                    T s = 0;
                    for (int dj = 0; dj < 2; dj++)
                        for (int di = 0; di < 2; di++) {
                            const int i = 2 * I + di, j = 2 * J + dj;
                            s += op_resid(c, zrow(q, j) + i, brow(q, j)[i], m, i, j);
                        }
                    bd[I] = T(0.25) * s;
                }
                __syncwarp();
                for (int d = -reach; d <= reach; d++) {
                    const int t = r + d;
                    if (d == 0 || t < 0 || t >= CS) continue;
                    const int tlo = t * ch, thi = tlo + ch;
                    if (!((J < tlo && J >= tlo - 4) || (J >= thi && J < thi + 4))) continue;
                    T* dst = cl_map(sm + st.ob[q + 1] + (J - tlo + G) * cm, t);
                    for (int I = lane; I < cm; I += 32) dst[I] = bd[I];
                }
            }
        } else {
            // the residual of the last slab level to every CTA
            for (int j = lo + warp; j < hi; j += NW)
                for (int i = lane; i < m; i += 32) {
                    const T rv = op_resid(c, zrow(q, j) + i, brow(q, j)[i], m, i, j);
                    T* p = sm + st.ostage + j * m + i;
                    for (int t = 0; t < CS; t++) *cl_map(p, t) = rv;
                }
        }
        cl_arrive();
        cl_wait();
    }

    // ------------------------------------------------------- exact level
    {
        const int q = st.nd - 1;
        const int m = st.lv[q].m, n = st.lv[q].n;
        const int dm = st.dl.m, dn = st.dl.n, N = dm * dn;
        const T* stg = sm + st.ostage;
        T* db = sm + st.odb;
        T* dz = sm + st.odz;
        for (int k = threadIdx.x; k < N; k += CL_THREADS) {
            const int J = k / dm, I = k - J * dm;
            T s = 0;
            for (int dj = 0; dj < 2; dj++)
                for (int di = 0; di < 2; di++) s += stg[(2 * J + dj) * m + 2 * I + di];
            db[k] = T(0.25) * s;
        }
        __syncthreads();
        // the rows of the exact solution this CTA's prolongation reads
        const int h = st.h[q], lo = r * h, hi = lo + h;
        const int J0 = max(0, (max(lo - 4, 0) >> 1) - 1);
        const int J1 = min(dn, ((min(hi + 4, n) - 1) >> 1) + 2);
        for (int row = J0 * dm + warp; row < J1 * dm; row += NW) {
            T s = 0;
            for (int k = lane; k < N; k += 32) s += st.dinv[size_t(row) * N + k] * db[k];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) dz[row] = s;
        }
        __syncthreads();
    }

    // ------------------------------------------------------------------ up
    for (int q = st.nd - 1; q >= 0; q--) {
        const CCc<T>& c = st.lv[q];
        const int m = c.m, h = st.h[q], lo = r * h, hi = lo + h;
        const int a = max(0, lo - 4), b = min(c.n, hi + 4);
        // pre-smoothed values (own rows, or the other CTAs' final rows) plus
        // the prolonged coarse correction, on the rows the four phases read
        auto correct = [&](auto row) {
            for (int j = a + warp; j < b; j += NW) {
                T* zr = zrow(q, j);
                const T* base = (j >= lo && j < hi) ? zr : sm + st.opre[q] + (j < lo ? j - (lo - 4) : 4 + (j - hi)) * m;
                for (int i = lane; i < m; i += 32) zr[i] = base[i] + cc_interp_rows(c, row, i, j);
            }
        };
        if (q == st.nd - 1) {
            const T* dz = sm + st.odz;
            const int dm = st.dl.m;
            correct([&](int J) -> const T* { return dz + J * dm; });
        } else {
            const int cm = st.lv[q + 1].m, ch = st.h[q + 1], clo = r * ch, chi = clo + ch;
            correct([&](int J) -> const T* {
                if (J >= clo && J < chi) return zrow(q + 1, J);
                return sm + st.opost[q + 1] + (J < clo ? J - (clo - 3) : 3 + (J - chi)) * cm;
            });
        }
        __syncthreads();
        phase(q, 1, lo - 3, hi + 3);
        phase(q, 0, lo - 2, hi + 2);
        phase(q, 1, lo - 1, hi + 1);
        phase(q, 0, lo, hi);
        if (q > 0) {
            for (int j = lo + warp; j < hi; j += NW) cl_push_row(sm, st.opost[q], zrow(q, j), m, j, r, h, CS, 3);
            cl_arrive();
            cl_wait();
        } else {
            for (int j = lo + warp; j < hi; j += NW) {
                const T* zr = zrow(0, j);
                for (int i = lane; i < m; i += 32) gz[i + size_t(m) * j] = zr[i];
            }
        }
    }
}

template <typename T>
int launch_cc_cluster(cudaStream_t s, const CCClusterArgs<T>& a, size_t smem, const T* b, T* z, int zero_init) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(a.cs));
    cfg.blockDim = dim3(CL_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = unsigned(a.cs);
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    VDI_CUDA(cudaLaunchKernelEx(&cfg, cc_cluster_cycle<T>, a, b, z, zero_init));
    return VDI_OK;
}

template <typename T>
cudaError_t cc_cluster_attr() {
    cudaError_t e = cudaFuncSetAttribute(cc_cluster_cycle<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(CL_SMEM_LIMIT));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(cc_cluster_cycle<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return e;
}

/** Clusters of `cs` CTAs with `smem` bytes each that the GPU can hold at
 * once (0: the launch would fail). */
template <typename T>
int cc_cluster_fits(int cs, size_t smem) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(cs));
    cfg.blockDim = dim3(CL_THREADS);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = unsigned(cs);
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, cc_cluster_cycle<T>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}
