/* gsl_shim.c -- implementations behind gsl/gsl_shim.h for the reference
 * build used as a checker (oracle/_ref).  They call the oracle's own
 * restatements (oracle/setup.c) of the same mathematics. */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gsl/gsl_shim.h"
#include "../oracle.h"

gsl_vector *gsl_vector_alloc(size_t n)
{
    gsl_vector *v = (gsl_vector *)malloc(sizeof(gsl_vector));
    v->size = n;
    v->stride = 1;
    v->data = (double *)malloc(sizeof(double) * (n ? n : 1));
    return v;
}

gsl_vector *gsl_vector_calloc(size_t n)
{
    gsl_vector *v = gsl_vector_alloc(n);
    memset(v->data, 0, sizeof(double) * (n ? n : 1));
    return v;
}

void gsl_vector_free(gsl_vector *v)
{
    if (v) {
        free(v->data);
        free(v);
    }
}

double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i * v->stride]; }
void gsl_vector_set(gsl_vector *v, size_t i, double x) { v->data[i * v->stride] = x; }

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2)
{
    gsl_matrix *m = (gsl_matrix *)malloc(sizeof(gsl_matrix));
    m->size1 = n1;
    m->size2 = n2;
    m->tda = n2;
    m->data = (double *)malloc(sizeof(double) * (n1 * n2 ? n1 * n2 : 1));
    return m;
}

void gsl_matrix_free(gsl_matrix *m)
{
    if (m) {
        free(m->data);
        free(m);
    }
}

double gsl_sf_legendre_sphPlm(int l, int m, double x) { return orc_sphPlm(l, m, x); }

int gsl_linalg_QR_decomp(gsl_matrix *A, gsl_vector *tau)
{
    orc_householder_qr((int)A->size1, (int)A->size2, A->data, tau->data);
    return 0;
}

int gsl_linalg_QR_lssolve(const gsl_matrix *QR, const gsl_vector *tau, const gsl_vector *b, gsl_vector *x,
                          gsl_vector *residual)
{
    /* residual holds the transformed right-hand side, as GSL's does */
    memcpy(residual->data, b->data, sizeof(double) * b->size);
    orc_householder_lssolve((int)QR->size1, (int)QR->size2, QR->data, tau->data, residual->data, x->data);
    return 0;
}

gsl_integration_glfixed_table *gsl_integration_glfixed_table_alloc(size_t n)
{
    gsl_integration_glfixed_table *t = (gsl_integration_glfixed_table *)malloc(sizeof(*t));
    t->n = n;
    t->x = (double *)malloc(sizeof(double) * n);
    t->w = (double *)malloc(sizeof(double) * n);
    orc_gauss_legendre((int)n, t->x, t->w);
    return t;
}

int gsl_integration_glfixed_point(double a, double b, size_t i, double *xi, double *wi,
                                  const gsl_integration_glfixed_table *t)
{
    const double half = 0.5 * (b - a), mid = 0.5 * (b + a);
    *xi = mid + half * t->x[i];
    *wi = half * t->w[i];
    return 0;
}
