/* gsl_spline.h -- stand-in for the GSL interpolation routines ic_basic.hpp
 * calls (TEST INFRASTRUCTURE ONLY; GSL is not part of the reference tree).
 * Only the natural cubic spline (gsl_interp_cspline) is provided: second
 * derivative zero at both ends, second-derivative halves from the tridiagonal
 * system of the interior knots (Thomas algorithm), evaluation as
 * y_i + t (b_i + t (c_i + t d_i)) on the interval x_i <= x < x_{i+1} found by
 * bisection.  The coefficients agree with GSL's to rounding.  Evaluating
 * outside [x_0, x_{n-1}] returns NaN (GSL reports a domain error). */
#ifndef GEV_REFSHIM_GSL_SPLINE_H
#define GEV_REFSHIM_GSL_SPLINE_H

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { int kind; } gsl_interp_type;
static const gsl_interp_type gev_shim_cspline_type = {1};
static const gsl_interp_type * gsl_interp_cspline = &gev_shim_cspline_type;

typedef struct { size_t last; } gsl_interp_accel;

typedef struct
{
	double * x;
	double * y;
	size_t size;
	double * b;
	double * c;
	double * d;
} gsl_spline;

static inline gsl_interp_accel * gsl_interp_accel_alloc(void) { return (gsl_interp_accel *) calloc(1, sizeof(gsl_interp_accel)); }
static inline void gsl_interp_accel_free(gsl_interp_accel * a) { free(a); }
static inline int gsl_interp_accel_reset(gsl_interp_accel * a) { if (a) a->last = 0; return 0; }

static inline gsl_spline * gsl_spline_alloc(const gsl_interp_type * t, size_t n)
{
	(void) t;
	gsl_spline * s = (gsl_spline *) calloc(1, sizeof(gsl_spline));
	s->size = n;
	s->x = (double *) calloc(n, sizeof(double));
	s->y = (double *) calloc(n, sizeof(double));
	s->b = (double *) calloc(n, sizeof(double));
	s->c = (double *) calloc(n, sizeof(double));
	s->d = (double *) calloc(n, sizeof(double));
	return s;
}

static inline void gsl_spline_free(gsl_spline * s)
{
	if (!s) return;
	free(s->x); free(s->y); free(s->b); free(s->c); free(s->d);
	free(s);
}

static inline int gsl_spline_init(gsl_spline * s, const double * x, const double * y, size_t n)
{
	memcpy(s->x, x, n * sizeof(double));
	memcpy(s->y, y, n * sizeof(double));
	for (size_t i = 0; i < n; i++) { s->b[i] = 0; s->c[i] = 0; s->d[i] = 0; }
	if (n > 2)
	{
		double * cp = (double *) calloc(n, sizeof(double));
		double * dp = (double *) calloc(n, sizeof(double));
		for (size_t i = 1; i + 1 < n; i++)
		{
			double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
			double r = 3.0 * ((y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0);
			double m = 2.0 * (h0 + h1) - (i > 1 ? h0 * cp[i - 1] : 0.0);
			cp[i] = h1 / m;
			dp[i] = (r - (i > 1 ? h0 * dp[i - 1] : 0.0)) / m;
		}
		for (size_t i = n - 2; i >= 1; i--)
		{
			s->c[i] = dp[i] - (i + 2 < n ? cp[i] * s->c[i + 1] : 0.0);
			if (i == 1) break;
		}
		free(cp);
		free(dp);
	}
	for (size_t i = 0; i + 1 < n; i++)
	{
		double h = x[i + 1] - x[i];
		s->b[i] = (y[i + 1] - y[i]) / h - h * (s->c[i + 1] + 2.0 * s->c[i]) / 3.0;
		s->d[i] = (s->c[i + 1] - s->c[i]) / (3.0 * h);
	}
	return 0;
}

static inline size_t gev_shim_spline_interval(const gsl_spline * s, double v)
{
	size_t lo = 0, hi = s->size - 1;
	while (hi > lo + 1)
	{
		size_t mid = (lo + hi) / 2;
		if (s->x[mid] > v) hi = mid; else lo = mid;
	}
	return lo;
}

static inline double gsl_spline_eval(const gsl_spline * s, double v, gsl_interp_accel * a)
{
	(void) a;
	if (!(v >= s->x[0] && v <= s->x[s->size - 1])) return NAN;
	size_t i = gev_shim_spline_interval(s, v);
	double t = v - s->x[i];
	return s->y[i] + t * (s->b[i] + t * (s->c[i] + t * s->d[i]));
}

static inline double gsl_spline_eval_deriv(const gsl_spline * s, double v, gsl_interp_accel * a)
{
	(void) a;
	if (!(v >= s->x[0] && v <= s->x[s->size - 1])) return NAN;
	size_t i = gev_shim_spline_interval(s, v);
	double t = v - s->x[i];
	return s->b[i] + t * (2.0 * s->c[i] + t * 3.0 * s->d[i]);
}

#endif
