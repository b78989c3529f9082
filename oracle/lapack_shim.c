/* Test infrastructure: routes the reference's `dsyev_` (scfcalculation.cpp:186-197, linked with
 * -llapack in src/common/makefile:83) to the LAPACK inside SciPy's bundled OpenBLAS, whose
 * exported names carry a `scipy_` prefix (32-bit integer ABI). */
extern void scipy_dsyev_(char *jobz, char *uplo, int *n, double *a, int *lda, double *w,
                         double *work, int *lwork, int *info);

void dsyev_(char *jobz, char *uplo, int *n, double *a, int *lda, double *w, double *work,
            int *lwork, int *info) {
  scipy_dsyev_(jobz, uplo, n, a, lda, w, work, lwork, info);
}
