/* Minimal GSL stand-ins for building GIZMO as a CPU oracle (test infrastructure).
 * Random numbers come from splitmix64, not GSL's ranlxd1; linear algebra,
 * eigen-solvers and quadrature are only reached by modules that the oracle
 * configuration never runs, and report failure if they are. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "gsl/gsl_eigen.h"
#include "gsl/gsl_errno.h"
#include "gsl/gsl_integration.h"
#include "gsl/gsl_linalg.h"
#include "gsl/gsl_randist.h"
#include "gsl/gsl_rng.h"
#include "gsl/gsl_sf_gamma.h"

static const gsl_rng_type ranlxd1_type = {1};
const gsl_rng_type *gsl_rng_ranlxd1 = &ranlxd1_type;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *t) { (void)t; gsl_rng *r = calloc(1, sizeof *r); r->state = 1; return r; }
void gsl_rng_free(gsl_rng *r) { free(r); }
void gsl_rng_set(gsl_rng *r, unsigned long seed) { r->state = seed ? seed : 1; }
static unsigned long long next64(gsl_rng *r)
{
    unsigned long long z = (r->state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double gsl_rng_uniform(gsl_rng *r) { return (next64(r) >> 11) * (1.0 / 9007199254740992.0); }
size_t gsl_rng_size(const gsl_rng *r) { (void)r; return sizeof(unsigned long long); }
void *gsl_rng_state(const gsl_rng *r) { return (void *)&r->state; }
double gsl_ran_ugaussian(gsl_rng *r)
{
    double u = gsl_rng_uniform(r), v = gsl_rng_uniform(r);
    if (u < 1e-300) u = 1e-300;
    return sqrt(-2 * log(u)) * cos(6.283185307179586 * v);
}
double gsl_ran_gaussian(gsl_rng *r, double sigma) { return sigma * gsl_ran_ugaussian(r); }
unsigned int gsl_ran_poisson(gsl_rng *r, double mu)
{
    double L = exp(-mu), p = 1;
    unsigned k = 0;
    do { k++; p *= gsl_rng_uniform(r); } while (p > L && k < 100000);
    return k - 1;
}
gsl_error_handler_t *gsl_set_error_handler_off(void) { return NULL; }
gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n)
{ gsl_integration_workspace *w = malloc(sizeof *w); w->limit = n; return w; }
void gsl_integration_workspace_free(gsl_integration_workspace *w) { free(w); }
int gsl_integration_qag(const gsl_function *f, double a, double b, double epsabs, double epsrel, size_t limit, int key,
                        gsl_integration_workspace *w, double *result, double *abserr)
{
    /* composite Simpson with 20000 panels: enough for the smooth drift/cooling integrands */
    (void)epsabs; (void)epsrel; (void)limit; (void)key; (void)w;
    int n = 20000;
    double h = (b - a) / n, s = f->function(a, f->params) + f->function(b, f->params);
    for (int i = 1; i < n; i++) s += (i & 1 ? 4 : 2) * f->function(a + i * h, f->params);
    *result = s * h / 3;
    if (abserr) *abserr = 0;
    return 0;
}
gsl_vector *gsl_vector_alloc(size_t n) { gsl_vector *v = malloc(sizeof *v); v->size = n; v->data = calloc(n, 8); v->owner = 1; return v; }
void gsl_vector_free(gsl_vector *v) { if (v) { if (v->owner) free(v->data); free(v); } }
double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i]; }
gsl_vector_view gsl_vector_view_array(double *base, size_t n) { gsl_vector_view r; r.vector.size = n; r.vector.data = base; r.vector.owner = 0; return r; }
gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2) { gsl_matrix *m = malloc(sizeof *m); m->size1 = n1; m->size2 = n2; m->data = calloc(n1 * n2, 8); m->owner = 1; return m; }
void gsl_matrix_free(gsl_matrix *m) { if (m) { if (m->owner) free(m->data); free(m); } }
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->size2 + j]; }
gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2) { gsl_matrix_view r; r.matrix.size1 = n1; r.matrix.size2 = n2; r.matrix.data = base; r.matrix.owner = 0; return r; }
static int unsupported(const char *w) { fprintf(stderr, "gsl shim: %s not available in the oracle build\n", w); return GSL_FAILURE; }
gsl_eigen_symm_workspace *gsl_eigen_symm_alloc(size_t n) { gsl_eigen_symm_workspace *w = malloc(sizeof *w); w->n = n; return w; }
void gsl_eigen_symm_free(gsl_eigen_symm_workspace *w) { free(w); }
int gsl_eigen_symm(gsl_matrix *A, gsl_vector *e, gsl_eigen_symm_workspace *w) { (void)A; (void)e; (void)w; return unsupported("gsl_eigen_symm"); }
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n) { gsl_eigen_symmv_workspace *w = malloc(sizeof *w); w->n = n; return w; }
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w) { free(w); }
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *e, gsl_matrix *v, gsl_eigen_symmv_workspace *w) { (void)A; (void)e; (void)v; (void)w; return unsupported("gsl_eigen_symmv"); }
gsl_permutation *gsl_permutation_alloc(size_t n) { gsl_permutation *p = malloc(sizeof *p); p->size = n; p->data = calloc(n, sizeof(size_t)); return p; }
void gsl_permutation_free(gsl_permutation *p) { if (p) { free(p->data); free(p); } }
int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *s) { (void)A; (void)p; (void)s; return unsupported("gsl_linalg_LU_decomp"); }
int gsl_linalg_LU_solve(const gsl_matrix *LU, const gsl_permutation *p, const gsl_vector *b, gsl_vector *x) { (void)LU; (void)p; (void)b; (void)x; return unsupported("gsl_linalg_LU_solve"); }
double gsl_sf_gamma(double x) { return tgamma(x); }
