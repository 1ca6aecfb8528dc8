/* The reference's inverse 3-D transform (A_k2a, fft_wrapper.h:662-681, Ooura
 * branch) on a k-space field read from a file: conjugate and scale by
 * 2/(NX NY NZ), rdft3dsort(-1), rdft3d(-1), both from the reference's own
 * fftsg3d.c.  Test infrastructure: pins the oracle's reading of the packed
 * kz = 0 / kz = NZ/2 planes.
 *
 *   ooura_inverse NX NY NZ in.bin out.bin
 * in.bin: complex128 [NX][NY][NZ/2+1]; out.bin: float64 [NX][NY][NZ+2]
 * (real field in the first NZ of each row).  Sizes are powers of two. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

void rdft3d(int, int, int, int, double ***, double *, int *, double *);
void rdft3dsort(int, int, int, int, double ***);

int main(int argc, char **argv) {
    if (argc != 6) return 2;
    const int    nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]), nz_ = nz + 2;
    const size_t n  = (size_t)nx * ny * nz_;
    double      *buf = malloc(sizeof(double) * n);
    FILE        *f   = fopen(argv[4], "rb");
    if (!buf || !f || fread(buf, sizeof(double), n, f) != n) return 1;
    fclose(f);
    const double scale = 2.0 / ((double)nx * ny * nz);
    for (size_t q = 0; q < n / 2; q++) buf[2 * q] *= scale, buf[2 * q + 1] *= -scale;
    double ***a = malloc(sizeof(double **) * nx);
    for (int i = 0; i < nx; i++) {
        a[i] = malloc(sizeof(double *) * ny);
        for (int j = 0; j < ny; j++) a[i][j] = buf + ((size_t)i * ny + j) * nz_;
    }
    int nt = nx > ny ? nx : ny;
    if (nz / 2 > nt) nt = nz / 2;
    int    *ip = calloc(2 + (size_t)sqrt((double)nt) + 8, sizeof(int));
    double *w  = calloc((size_t)nt * 3 / 2 + 8, sizeof(double));
    double *t  = calloc((size_t)32 * (nx > ny ? nx : ny), sizeof(double));
    rdft3dsort(nx, ny, nz, -1, a);
    rdft3d(nx, ny, nz, -1, a, t, ip, w);
    f = fopen(argv[5], "wb");
    if (!f || fwrite(buf, sizeof(double), n, f) != n) return 1;
    fclose(f);
    return 0;
}
