/* Minimal CBLAS declaration for building the reference CCD sources against the OpenBLAS
 * that ships inside scipy (it exports its CBLAS entry points with a "scipy_" prefix).
 *
 * Test infrastructure only.  The reference calls only cblas_dgemm with row-major,
 * no-transpose operands (calc.cpp:146,167,188,277,298, MBPT2Corr.cpp:86).  The enum
 * values are the standard CBLAS ones.
 */
#ifndef CCD_ORACLE_CBLAS_SHIM_H
#define CCD_ORACLE_CBLAS_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };

void scipy_cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                       int m, int n, int k, double alpha, const double *a, int lda,
                       const double *b, int ldb, double beta, double *c, int ldc);
void scipy_openblas_set_num_threads(int n);

#define cblas_dgemm scipy_cblas_dgemm

#ifdef __cplusplus
}
#endif

#endif
