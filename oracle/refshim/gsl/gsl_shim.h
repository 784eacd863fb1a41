/* gsl_shim.h -- the part of the GSL interface that closures-2d's sources use
 * (utils.cpp:55-60, momopt_init.cpp:97-265, moment_init.cpp, dn_init.cpp),
 * declared for building the reference as a checker (oracle/_ref).  The
 * implementations (gsl_shim.c) are this project's own from the mathematics:
 * Gauss-Legendre by Newton on the Legendre recurrence, the normalised
 * associated Legendre function with the Condon-Shortley phase, Householder
 * QR least squares.  Test infrastructure; nothing in the product links it. */
#ifndef CLOSURES_GSL_SHIM_H
#define CLOSURES_GSL_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct {
    size_t size;
    size_t stride;
    double *data;
} gsl_vector;
typedef struct {
    size_t size1, size2, tda;
    double *data;
} gsl_matrix;
typedef struct {
    size_t n;
    double *x, *w;   /* nodes ascending on [-1, 1] and weights */
} gsl_integration_glfixed_table;

gsl_vector *gsl_vector_alloc(size_t n);
gsl_vector *gsl_vector_calloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);
gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
double gsl_sf_legendre_sphPlm(int l, int m, double x);
int gsl_linalg_QR_decomp(gsl_matrix *A, gsl_vector *tau);
int gsl_linalg_QR_lssolve(const gsl_matrix *QR, const gsl_vector *tau, const gsl_vector *b, gsl_vector *x,
                          gsl_vector *residual);
gsl_integration_glfixed_table *gsl_integration_glfixed_table_alloc(size_t n);
int gsl_integration_glfixed_point(double a, double b, size_t i, double *xi, double *wi,
                                  const gsl_integration_glfixed_table *t);
#ifdef __cplusplus
}
#endif
#endif
