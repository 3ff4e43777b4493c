#ifndef GG_SHIM_GSL_EIGEN_H
#define GG_SHIM_GSL_EIGEN_H
#include "gsl_vector.h"
typedef struct { size_t n; } gsl_eigen_symm_workspace;
typedef struct { size_t n; } gsl_eigen_symmv_workspace;
gsl_eigen_symm_workspace *gsl_eigen_symm_alloc(size_t n);
void gsl_eigen_symm_free(gsl_eigen_symm_workspace *w);
int gsl_eigen_symm(gsl_matrix *A, gsl_vector *eval, gsl_eigen_symm_workspace *w);
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n);
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w);
#endif
