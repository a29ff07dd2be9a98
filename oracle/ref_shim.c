/*
 * Two f2c runtime helpers that the reference's built-in BLAS declares
 * (complex modulus, used only by crotg/zrotg, off the factorization path)
 * but whose definitions live outside the reference tree.  Defined here so
 * the reference library loads with every symbol resolved.  Test
 * infrastructure only.
 */
#include <math.h>
typedef struct { float r, i; } ref_complex;
typedef struct { double r, i; } ref_doublecomplex;
double c_f2c_abs(ref_complex *z) { return hypot((double)z->r, (double)z->i); }
double z_f2c_abs(ref_doublecomplex *z) { return hypot(z->r, z->i); }
