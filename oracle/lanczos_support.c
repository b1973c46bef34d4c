/* Support routines of the translated SPRLAN build (TEST INFRASTRUCTURE ONLY:
 * linked into oracle/_ref/libsprref.so, never into the product).
 *
 * SPRLAN (src/SPR/sprlan.f) calls four level-1 BLAS routines and one SAM
 * group-0 utility that the oracle build does not translate:
 *   DCOPY, DSCAL, DDOT, DAXPY : the reference BLAS definitions (Netlib
 *     level-1: strides may be zero or negative, a negative stride starts
 *     from the far end); INTEGER arguments are 32-bit, as SPRLAN passes
 *     them (its `_i4` literals and INTEGER(kind=i4) variables);
 *   IMP(3) (src/Mdr.f): the number of significant decimal digits, i.e. the
 *     largest i with 1 + 10^-i > 1 (15 for IEEE double), 0 for other
 *     arguments (the reference routine keeps AUX in a COMMON block, which
 *     the translator does not take).
 * The SAM group routines are built without -fdefault-integer-8 in the
 * reference (only SPR is I8), so their INTEGERs are 32-bit here too. */
#include <stdint.h>

static int64_t first(int32_t n, int32_t inc) { return inc < 0 ? (int64_t)(1 - n) * inc : 0; }

void dcopy_(const int32_t *n, const double *x, const int32_t *incx, double *y, const int32_t *incy) {
    int64_t ix = first(*n, *incx), iy = first(*n, *incy);
    for (int32_t i = 0; i < *n; ++i, ix += *incx, iy += *incy) y[iy] = x[ix];
}

void dscal_(const int32_t *n, const double *a, double *x, const int32_t *incx) {
    if (*incx <= 0) return;
    for (int64_t i = 0, ix = 0; i < *n; ++i, ix += *incx) x[ix] = *a * x[ix];
}

double ddot_(const int32_t *n, const double *x, const int32_t *incx, const double *y, const int32_t *incy) {
    double s = 0.0;
    int64_t ix = first(*n, *incx), iy = first(*n, *incy);
    for (int32_t i = 0; i < *n; ++i, ix += *incx, iy += *incy) s += x[ix] * y[iy];
    return s;
}

void daxpy_(const int32_t *n, const double *a, const double *x, const int32_t *incx, double *y,
            const int32_t *incy) {
    if (*n <= 0 || *a == 0.0) return;
    int64_t ix = first(*n, *incx), iy = first(*n, *incy);
    for (int32_t i = 0; i < *n; ++i, ix += *incx, iy += *incy) y[iy] = y[iy] + *a * x[ix];
}

int32_t imp_(const int32_t *num) {
    if (*num != 3) return 0;
    volatile double eps = 1.0, aux;
    for (int32_t i = 1; i <= 50; ++i) {
        eps = eps / 10.0;
        aux = 1.0 + eps;
        if (!(aux > 1.0)) return i - 1;
    }
    return 0;
}
