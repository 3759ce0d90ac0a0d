/* Declarations for the Numerical-Recipes style Jacobi eigen-solver that the
 * plastic and visco-plastic hooks carry (plastic/Constitutive.c:249-480).
 * ROTATE is the standard Jacobi plane-rotation update (Press et al.,
 * Numerical Recipes in C, 2nd ed., section 11.1), restated here. */
#ifndef SNAC_SHIM_NR_H
#define SNAC_SHIM_NR_H
#define ROTATE(a, i, j, k, l) g = a[i][j]; h = a[k][l]; a[i][j] = g - s * (h + g * tau); a[k][l] = h + s * (g - h * tau);
#define NR_END 1
#define FREE_ARG char*
double** dmatrix(long nrl, long nrh, long ncl, long nch);
double* dvector(long nl, long nh);
int* ivector(long nl, long nh);
void free_ivector(int* v, long nl, long nh);
void free_dmatrix(double** m, long nrl, long nrh, long ncl, long nch);
void free_dvector(double* v, long nl, long nh);
void nrerror(char error_text[]);
int jacobi(double** a, double* d, double** v);
int eigsrt(double* d, double** v);
#endif
