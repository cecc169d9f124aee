/*
 * Test infrastructure (oracle only): a minimal stand-in for the three Intel MKL
 * names the reference's built sources use -- MKL_Complex16, vdAdd and vzAdd
 * (src/lib/derivatives.c:1250,3050).  MKL is not installed here.  The
 * semantics follow MKL's published vector-math reference:
 *   vdAdd(n, a, b, r): r[i] = a[i] + b[i] for 0 <= i < n (double)
 *   vzAdd(n, a, b, r): the same for complex doubles, component-wise.
 */
#ifndef UPH_ORACLE_MKL_SHIM_H
#define UPH_ORACLE_MKL_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
typedef struct { double real; double imag; } MKL_Complex16;
void vdAdd(const int n, const double *a, const double *b, double *r);
void vzAdd(const int n, const MKL_Complex16 *a, const MKL_Complex16 *b, MKL_Complex16 *r);
#ifdef __cplusplus
}
#endif
#endif
