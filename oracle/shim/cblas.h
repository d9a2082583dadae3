/* Oracle build shim: CBLAS prototypes for the compiled reference library.
 *
 * Test infrastructure only. The reference sources include <cblas.h>; this
 * header maps the calls they make onto the OpenBLAS copy bundled with SciPy,
 * which exports every CBLAS symbol with a "scipy_" prefix. Only the enum
 * values and prototypes the reference actually calls are declared. */
#ifndef ORACLE_SHIM_CBLAS_H
#define ORACLE_SHIM_CBLAS_H
#include <complex.h>

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;

#define SHIM_BLAS(name) scipy_##name
#define cblas_dgemm SHIM_BLAS(cblas_dgemm)
#define cblas_sgemm SHIM_BLAS(cblas_sgemm)
#define cblas_cgemm SHIM_BLAS(cblas_cgemm)
#define cblas_zgemm SHIM_BLAS(cblas_zgemm)
#define cblas_dnrm2 SHIM_BLAS(cblas_dnrm2)
#define cblas_snrm2 SHIM_BLAS(cblas_snrm2)
#define cblas_dznrm2 SHIM_BLAS(cblas_dznrm2)
#define cblas_scnrm2 SHIM_BLAS(cblas_scnrm2)
#define cblas_daxpy SHIM_BLAS(cblas_daxpy)
#define cblas_saxpy SHIM_BLAS(cblas_saxpy)
#define cblas_caxpy SHIM_BLAS(cblas_caxpy)
#define cblas_zaxpy SHIM_BLAS(cblas_zaxpy)
#define cblas_dcopy SHIM_BLAS(cblas_dcopy)
#define cblas_scopy SHIM_BLAS(cblas_scopy)
#define cblas_ccopy SHIM_BLAS(cblas_ccopy)
#define cblas_zcopy SHIM_BLAS(cblas_zcopy)
#define cblas_dscal SHIM_BLAS(cblas_dscal)
#define cblas_sscal SHIM_BLAS(cblas_sscal)
#define cblas_cscal SHIM_BLAS(cblas_cscal)
#define cblas_zscal SHIM_BLAS(cblas_zscal)
#define cblas_ddot SHIM_BLAS(cblas_ddot)

void cblas_dgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
        int, int, int, double, const double *, int, const double *, int,
        double, double *, int);
void cblas_sgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
        int, int, int, float, const float *, int, const float *, int,
        float, float *, int);
void cblas_cgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
        int, int, int, const void *, const void *, int, const void *, int,
        const void *, void *, int);
void cblas_zgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
        int, int, int, const void *, const void *, int, const void *, int,
        const void *, void *, int);
double cblas_dnrm2(int, const double *, int);
float cblas_snrm2(int, const float *, int);
double cblas_dznrm2(int, const void *, int);
float cblas_scnrm2(int, const void *, int);
void cblas_daxpy(int, double, const double *, int, double *, int);
void cblas_saxpy(int, float, const float *, int, float *, int);
void cblas_caxpy(int, const void *, const void *, int, void *, int);
void cblas_zaxpy(int, const void *, const void *, int, void *, int);
void cblas_dcopy(int, const double *, int, double *, int);
void cblas_scopy(int, const float *, int, float *, int);
void cblas_ccopy(int, const void *, int, void *, int);
void cblas_zcopy(int, const void *, int, void *, int);
void cblas_dscal(int, double, double *, int);
void cblas_sscal(int, float, float *, int);
void cblas_cscal(int, const void *, void *, int);
void cblas_zscal(int, const void *, void *, int);
double cblas_ddot(int, const double *, int, const double *, int);
#endif
