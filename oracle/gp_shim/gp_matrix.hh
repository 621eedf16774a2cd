// ORACLE TEST INFRASTRUCTURE — not part of the product.
//
// Clean-room stand-in for the gp_matrix class of the absent utils-gp library,
// with only what the reference's analysis tool uses (tt_analysis.cc:104-146:
// the constructor from a file name and the members m, dx, x, f). It reads a
// Gnuplot binary matrix file as the reference writes one
// (gas_layer_solve.cc:258-282): float32 n, then n float32 x coordinates, then
// rows of one float32 y coordinate followed by n float32 values. The field
// values and coordinates are widened to double; dx is the mean spacing of x.
#ifndef VDI_GP_MATRIX_SHIM_HH
#define VDI_GP_MATRIX_SHIM_HH

#include <cstdio>
#include <cstdlib>
#include <vector>

class gp_matrix {
    public:
        /** The number of columns (x points) and rows (y points). */
        int m, n;
        /** The mean x spacing. */
        double dx;
        /** The x and y coordinates. */
        double *x, *y;
        /** The field values, row by row (m per row). */
        double *f;
        gp_matrix(const char* filename) : m(0), n(0), dx(0), x(NULL), y(NULL), f(NULL) {
            FILE* fp = fopen(filename, "rb");
            if (fp == NULL) {
                fprintf(stderr, "gp_matrix: cannot open %s\n", filename);
                exit(1);
            }
            float hdr;
            if (fread(&hdr, sizeof(float), 1, fp) != 1) bad(filename);
            m = int(hdr);
            if (m <= 0) bad(filename);
            std::vector<float> row(m + 1);
            row[0] = hdr;
            if (fread(&row[1], sizeof(float), m, fp) != size_t(m)) bad(filename);
            x = new double[m];
            for (int i = 0; i < m; i++) x[i] = row[i + 1];
            dx = m > 1 ? (x[m - 1] - x[0]) / (m - 1) : 1.0;
            std::vector<double> ys, fs;
            while (fread(&row[0], sizeof(float), m + 1, fp) == size_t(m + 1)) {
                ys.push_back(row[0]);
                for (int i = 0; i < m; i++) fs.push_back(row[i + 1]);
            }
            fclose(fp);
            n = int(ys.size());
            if (n == 0) bad(filename);
            y = new double[n];
            f = new double[size_t(m) * n];
            for (int j = 0; j < n; j++) y[j] = ys[j];
            for (size_t k = 0; k < fs.size(); k++) f[k] = fs[k];
        }
        ~gp_matrix() {
            delete[] x;
            delete[] y;
            delete[] f;
        }
    private:
        static void bad(const char* filename) {
            fprintf(stderr, "gp_matrix: malformed file %s\n", filename);
            exit(1);
        }
};

#endif
