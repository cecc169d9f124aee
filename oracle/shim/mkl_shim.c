/*
 * Test infrastructure (oracle only): element-wise vector addition used by the
 * compiled reference in place of Intel MKL (not installed here).  Each output
 * element is the single IEEE-754 double addition a[i] + b[i], which is what
 * MKL's vdAdd computes in its default (high-accuracy) mode.
 */
#include "mkl.h"

void vdAdd(const int n, const double *a, const double *b, double *r)
{
  for (int i = 0; i < n; i++)
    r[i] = a[i] + b[i];
}

void vzAdd(const int n, const MKL_Complex16 *a, const MKL_Complex16 *b, MKL_Complex16 *r)
{
  for (int i = 0; i < n; i++) {
    r[i].real = a[i].real + b[i].real;
    r[i].imag = a[i].imag + b[i].imag;
  }
}
