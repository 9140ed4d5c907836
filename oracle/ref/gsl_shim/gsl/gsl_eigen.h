/* Stand-in for the names the reference's sources.c uses to orient plane
 * sources (solve_u_v(), sources.c:80-102). The oracle harness builds no
 * plane sources: the bodies in gsl_shim.c stop the process if reached. */
#ifndef ORACLE_GSL_EIGEN_H
#define ORACLE_GSL_EIGEN_H
#include <stddef.h>
typedef struct { size_t size1, size2; double *data; } gsl_matrix;
typedef struct { size_t size; double *data; } gsl_vector;
typedef struct { gsl_matrix matrix; } gsl_matrix_view;
typedef struct { gsl_vector vector; } gsl_vector_view;
typedef struct { int unused; } gsl_eigen_symmv_workspace;
#define GSL_EIGEN_SORT_ABS_ASC 0
gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2);
gsl_vector *gsl_vector_alloc(size_t n);
gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n);
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv_sort(gsl_vector *eval, gsl_matrix *evec, int type);
gsl_vector_view gsl_matrix_column(gsl_matrix *m, size_t j);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_matrix_free(gsl_matrix *m);
void gsl_vector_free(gsl_vector *v);
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w);
#endif
