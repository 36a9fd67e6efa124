/* The BR values-only solver under its LAPACK names.
 *
 * The reference's BR routine was upstreamed to Reference-LAPACK as
 * DSTEBR / SSTEBR with LAPACKE wrappers (README.md:13); that interface is
 * not part of the reference tree, whose routine is DSTEDC_DC_BR
 * (cpu/src/dstedc_dc_br.f:7).  These entries keep DSTEDC_DC_BR's argument
 * list and semantics under the upstream names, so a LAPACK caller of either
 * links against libbrdc_b200.so unchanged:
 *
 *   N       order (INFO = -1 if N < 0)
 *   D       in: the diagonal; out: the eigenvalues in ascending order
 *   E       in: the N-1 off-diagonal entries; destroyed
 *   WORK    LWORK >= LWMIN = max(1, (16 + 2 NTHR) N) for N > 25, else 1
 *           (INFO = -5 if smaller); WORK(1) returns LWMIN
 *   IWORK   LIWORK >= LIWMIN = max(1, 7 N) for N > 25, else 1 (INFO = -7);
 *           IWORK(1) returns LIWMIN
 *   LWORK = -1 or LIWORK = -1 is a workspace query (dstedc_dc_br.f:44-75)
 *   INFO    0 on success; > 0 if a root did not converge (its position) or
 *           N + 1 if the GPU could not be used
 *
 * The solve runs on the GPU (host arrays copied in and out, device buffers
 * allocated per call); the host WORK and IWORK are only checked.  SSTEBR
 * solves in FP64 and rounds the eigenvalues to float.  Fortran calling
 * convention: every argument by reference.
 *
 * The LAPACKE forms follow LAPACKE's convention for values-only routines
 * (as LAPACKE_dsterf): arguments by value, INFO returned; the plain form
 * checks D and E for NaN (returns -2 / -3), queries and allocates the
 * workspace (returns -1010, LAPACK_WORK_MEMORY_ERROR, if it cannot).
 * brdc_dstedc_dc_br_ (brdc.h) is the same routine under the reference's
 * own name.
 */
#ifndef BRDC_LAPACK_H
#define BRDC_LAPACK_H

#ifdef __cplusplus
extern "C" {
#endif

void dstebr_(const int *n, double *d, double *e, double *work, const int *lwork,
             int *iwork, const int *liwork, int *info);
void sstebr_(const int *n, float *d, float *e, float *work, const int *lwork,
             int *iwork, const int *liwork, int *info);

int LAPACKE_dstebr(int n, double *d, double *e);
int LAPACKE_dstebr_work(int n, double *d, double *e, double *work, int lwork,
                        int *iwork, int liwork);
int LAPACKE_sstebr(int n, float *d, float *e);
int LAPACKE_sstebr_work(int n, float *d, float *e, float *work, int lwork,
                        int *iwork, int liwork);

#ifdef __cplusplus
}
#endif

#endif /* BRDC_LAPACK_H */
