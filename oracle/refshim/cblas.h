/*
 * cblas.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Stand-in for the three CBLAS routines the reference's headers name
 * (cblas_sdot at query.h:166,178; cblas_saxpy/cblas_snrm2 at
 * sc_algorithm.h:212-213).  The reference's OpenBLAS submodule is not
 * vendored, so the oracle build supplies these as plain sequential loops:
 * sdot is "s += x[i]*y[i]" in float, which fixes the summation order that
 * the oracle restatement and the GPU's exact table build both follow.
 */
#ifndef ORACLE_CBLAS_SHIM_H_
#define ORACLE_CBLAS_SHIM_H_
#include <math.h>

static inline float cblas_sdot(const int n, const float *x, const int incx,
                               const float *y, const int incy) {
    float s = 0.0f;
    for (int i = 0; i < n; i++) s += x[i * incx] * y[i * incy];
    return s;
}

static inline void cblas_saxpy(const int n, const float alpha, const float *x,
                               const int incx, float *y, const int incy) {
    for (int i = 0; i < n; i++) y[i * incy] += alpha * x[i * incx];
}

static inline float cblas_snrm2(const int n, const float *x, const int incx) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += (double)x[i * incx] * (double)x[i * incx];
    return (float)sqrt(s);
}
#endif
