/* Minimal stand-in for the GSL pieces GIZMO includes (test infrastructure). */
#ifndef GG_SHIM_GSL_MATH_H
#define GG_SHIM_GSL_MATH_H
#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
static inline double gsl_pow_2(double x) { return x * x; }
static inline double gsl_pow_3(double x) { return x * x * x; }
static inline double gsl_pow_4(double x) { double y = x * x; return y * y; }
static inline double gsl_pow_5(double x) { double y = x * x; return y * y * x; }
static inline double gsl_pow_int(double x, int n)
{
    double r = 1;
    int neg = n < 0;
    if (neg) n = -n;
    while (n) { if (n & 1) r *= x; x *= x; n >>= 1; }
    return neg ? 1.0 / r : r;
}
typedef struct { double (*function)(double x, void *params); void *params; } gsl_function;
#endif
