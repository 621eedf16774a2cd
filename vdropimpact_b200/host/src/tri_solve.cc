// tri_solve (tri_solve.cc:1-49) over the device tridiagonal solver.
#include "tri_solve.hh"

#include <cstdio>
#include <cstdlib>

#include <cuda_runtime.h>

#include "common.hh"
#include "vdi.h"

tri_solve::tri_solve(int m_)
    : m(m_), a(new double[4 * m_]()), b(a + m_), c(b + m_), d(c + m_), dev(NULL) {
    if (cudaMalloc(&dev, 4 * m * sizeof(double)) != cudaSuccess) fatal_error("tri_solve: cudaMalloc failed", 1);
}

tri_solve::~tri_solve() {
    cudaFree(dev);
    delete[] a;
}

void tri_solve::solve_lapack() {
    // a, b, c, d are contiguous (one 4m block, as the reference allocates)
    if (cudaMemcpy(dev, a, 4 * m * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        fatal_error("tri_solve: copy failed", 1);
    int pivoted = 0;
    int st = vdi_tri_solve(m, dev, dev + m, dev + 2 * m, dev + 3 * m, NULL, &pivoted);
    if (st == VDI_ERR_TRI_SINGULAR) {
        fputs("LAPACK routine failed\n", stderr);
        exit(1);
    }
    vdi_check(st, "vdi_tri_solve");
    if (cudaMemcpy(a, dev, 4 * m * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        fatal_error("tri_solve: copy failed", 1);
}

void tri_solve::solve() { solve_lapack(); }
