/* C caller of the drop-in ABI in the call pattern of the reference's
 * example_usage.c (single call, then preprocess once + solve) and of its
 * profiler (timed variants, PSTRSV_VERBOSE).  Builds the lower triangle of the
 * 5-point Poisson matrix on an N x N grid (or, with a third argument, reads the
 * lower triangle of a MatrixMarket file), b = L x_real with the reference's
 * known-answer x_real = (rand()%71)+1 + (i%1000)/10 (example_usage.c:81-85), and
 * prints the 2-norm error of each solve.  Exit status 0 when every error is
 * below the reference's 1e-4 acceptance threshold. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "spike_pstrsv.h"

static double err2(const double *x, const double *xr, int m) {
    double s = 0;
    for (int i = 0; i < m; i++) s += (x[i] - xr[i]) * (x[i] - xr[i]);
    return sqrt(s);
}

int main(int argc, char **argv) {
    const int N = argc > 1 ? atoi(argv[1]) : 64;
    const int P = argc > 2 ? atoi(argv[2]) : 4;
    int m = N * N;
    MKL_INT *ia, *ja;
    double *a;
    if (argc > 3) {
        /* the profiler's way in (runtime_analysis.c:290-292): a MatrixMarket file,
         * lower triangle */
        matrixMarketToCSR(argv[3], &a, &ia, &ja, &m, 'L', 'N');
        if (!a) return 2;
        printf("read %s: %d rows, %d entries\n", argv[3], m, ia[m]);
    } else {
        ia = malloc(sizeof(MKL_INT) * (m + 1));
        ja = malloc(sizeof(MKL_INT) * 3 * m);
        a = malloc(sizeof(double) * 3 * m);
        int q = 0;
        for (int i = 0; i < m; i++) {
            ia[i] = q;
            if (i >= N) { ja[q] = i - N; a[q++] = -1.0; }
            if (i % N) { ja[q] = i - 1; a[q++] = -1.0; }
            ja[q] = i; a[q++] = 4.0;
        }
        ia[m] = q;
    }
    double *xr = malloc(sizeof(double) * m), *b = calloc(m, sizeof(double));
    double *b2 = malloc(sizeof(double) * m), *x = calloc(m, sizeof(double));
    for (int i = 0; i < m; i++) xr[i] = ((rand() % 71) + 1) + ((double)(i % 1000) / 10.0);
    for (int i = 0; i < m; i++)
        for (int k = ia[i]; k < ia[i + 1]; k++) b[i] += a[k] * xr[ja[k]];
    int bad = 0;

    memcpy(b2, b, sizeof(double) * m);
    spike_pstrsv('L', m, a, ia, ja, b2, x, P);
    double e = err2(x, xr, m);
    printf("spike_pstrsv 2-norm error: %e\n", e);
    bad |= !(e <= 1e-4);

    memset(x, 0, sizeof(double) * m);
    spike_pstrsv_preproc(a, ia, ja, m, P, 'L');
    for (int rep = 0; rep < 3; rep++) {
        memcpy(b2, b, sizeof(double) * m);
        spike_pstrsv_solve('L', m, b2, x, P);
    }
    e = err2(x, xr, m);
    printf("preproc + solve 2-norm error: %e, reduced system %d rows\n", e, numRowsReducedSystem);
    bad |= !(e <= 1e-4);

    PSTRSV_VERBOSE = 1;
    _spike_pstrsv_preproc(a, ia, ja, m, P, 'L');
    PSTRSV_VERBOSE = 0;
    memcpy(b2, b, sizeof(double) * m);
    _spike_pstrsv_solve('L', m, b2, x, P);
    e = err2(x, xr, m);
    printf("timed: produceS %.6f s, computeY %.6f s, solveD2 %.6f s, error %e\n", produceS_timer_pstrsv3,
           computeY_timer[0], solveD2_timer[0], e);
    bad |= !(e <= 1e-4);
    free_PSTRSV3();
    free(ia); free(ja); free(a); free(xr); free(b); free(b2); free(x);
    return bad;
}
