#ifndef GG_SHIM_GSL_VECTOR_H
#define GG_SHIM_GSL_VECTOR_H
#include <stddef.h>
typedef struct { size_t size; double *data; int owner; } gsl_vector;
typedef struct { gsl_vector vector; } gsl_vector_view;
typedef struct { size_t size1, size2; double *data; int owner; } gsl_matrix;
typedef struct { gsl_matrix matrix; } gsl_matrix_view;
gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
gsl_vector_view gsl_vector_view_array(double *base, size_t n);
gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);
gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2);
#endif
