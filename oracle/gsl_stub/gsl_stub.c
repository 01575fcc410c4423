/* Aborting definitions for the GSL stub header (test infrastructure only). */
#include <stdio.h>
#include <stdlib.h>
#include "gsl/gsl_spline.h"

static void gsl_stub_abort(const char *what) {
  fprintf(stderr, "oracle gsl stub: %s called; the spline EoS is not supported\n", what);
  abort();
}
const gsl_interp_type *gsl_interp_cspline = 0;
gsl_interp_accel *gsl_interp_accel_alloc(void) { gsl_stub_abort("gsl_interp_accel_alloc"); return 0; }
gsl_spline *gsl_spline_alloc(const gsl_interp_type *t, size_t n) { (void)t; (void)n; gsl_stub_abort("gsl_spline_alloc"); return 0; }
int gsl_spline_init(gsl_spline *s, const double *x, const double *y, size_t n) { (void)s; (void)x; (void)y; (void)n; gsl_stub_abort("gsl_spline_init"); return 0; }
double gsl_spline_eval(const gsl_spline *s, double x, gsl_interp_accel *a) { (void)s; (void)x; (void)a; gsl_stub_abort("gsl_spline_eval"); return 0.; }
void gsl_spline_free(gsl_spline *s) { (void)s; gsl_stub_abort("gsl_spline_free"); }
void gsl_interp_accel_free(gsl_interp_accel *a) { (void)a; gsl_stub_abort("gsl_interp_accel_free"); }
