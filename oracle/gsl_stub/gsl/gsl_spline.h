/* Test-infrastructure stub: declares the handful of GSL spline names that the
 * reference's EoSs class (src/eos.cpp:27-119) refers to, so the reference hot
 * path links without GSL.  The oracle never constructs an EoSs object; every
 * stub definition (gsl_stub.c) aborts if it is ever called. */
#pragma once
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct gsl_interp_accel_stub gsl_interp_accel;
typedef struct gsl_spline_stub gsl_spline;
typedef struct gsl_interp_type_stub gsl_interp_type;
extern const gsl_interp_type *gsl_interp_cspline;
gsl_interp_accel *gsl_interp_accel_alloc(void);
gsl_spline *gsl_spline_alloc(const gsl_interp_type *t, size_t n);
int gsl_spline_init(gsl_spline *s, const double *x, const double *y, size_t n);
double gsl_spline_eval(const gsl_spline *s, double x, gsl_interp_accel *a);
void gsl_spline_free(gsl_spline *s);
void gsl_interp_accel_free(gsl_interp_accel *a);
#ifdef __cplusplus
}
#endif
