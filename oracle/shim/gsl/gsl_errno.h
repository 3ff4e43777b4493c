#ifndef GG_SHIM_GSL_ERRNO_H
#define GG_SHIM_GSL_ERRNO_H
#define GSL_SUCCESS 0
#define GSL_FAILURE (-1)
typedef void gsl_error_handler_t(const char *reason, const char *file, int line, int gsl_errno);
gsl_error_handler_t *gsl_set_error_handler_off(void);
#endif
