#ifndef GG_SHIM_GSL_SPLINE_H
#define GG_SHIM_GSL_SPLINE_H
typedef struct gsl_spline gsl_spline;
typedef struct gsl_interp_accel gsl_interp_accel;
#endif
