/* Oracle build shim: LAPACKE prototypes for the compiled reference library.
 *
 * Test infrastructure only; see cblas.h in this directory. Maps the LAPACKE
 * calls of the reference sources onto SciPy's bundled OpenBLAS ("scipy_"
 * prefixed exports, LP64 integers). */
#ifndef ORACLE_SHIM_LAPACKE_H
#define ORACLE_SHIM_LAPACKE_H
#include <complex.h>
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
typedef int lapack_int;
typedef float _Complex lapack_complex_float;
typedef double _Complex lapack_complex_double;

#define SHIM_LAPACKE(name) scipy_##name
#define LAPACKE_dgesdd SHIM_LAPACKE(LAPACKE_dgesdd)
#define LAPACKE_sgesdd SHIM_LAPACKE(LAPACKE_sgesdd)
#define LAPACKE_cgesdd SHIM_LAPACKE(LAPACKE_cgesdd)
#define LAPACKE_zgesdd SHIM_LAPACKE(LAPACKE_zgesdd)
#define LAPACKE_dgesdd_work SHIM_LAPACKE(LAPACKE_dgesdd_work)
#define LAPACKE_zgesdd_work SHIM_LAPACKE(LAPACKE_zgesdd_work)
#define LAPACKE_dgeqrf_work SHIM_LAPACKE(LAPACKE_dgeqrf_work)
#define LAPACKE_zgeqrf_work SHIM_LAPACKE(LAPACKE_zgeqrf_work)
#define LAPACKE_dorgqr_work SHIM_LAPACKE(LAPACKE_dorgqr_work)
#define LAPACKE_zungqr_work SHIM_LAPACKE(LAPACKE_zungqr_work)
#define LAPACKE_dgeqp3_work SHIM_LAPACKE(LAPACKE_dgeqp3_work)
#define LAPACKE_dlarnv_work SHIM_LAPACKE(LAPACKE_dlarnv_work)
#define LAPACKE_zlarnv_work SHIM_LAPACKE(LAPACKE_zlarnv_work)
#define LAPACKE_dpotrf SHIM_LAPACKE(LAPACKE_dpotrf)
#define LAPACKE_spotrf SHIM_LAPACKE(LAPACKE_spotrf)
#define LAPACKE_cpotrf SHIM_LAPACKE(LAPACKE_cpotrf)
#define LAPACKE_zpotrf SHIM_LAPACKE(LAPACKE_zpotrf)

lapack_int LAPACKE_dgesdd(int, char, lapack_int, lapack_int, double *,
        lapack_int, double *, double *, lapack_int, double *, lapack_int);
lapack_int LAPACKE_sgesdd(int, char, lapack_int, lapack_int, float *,
        lapack_int, float *, float *, lapack_int, float *, lapack_int);
lapack_int LAPACKE_cgesdd(int, char, lapack_int, lapack_int,
        lapack_complex_float *, lapack_int, float *, lapack_complex_float *,
        lapack_int, lapack_complex_float *, lapack_int);
lapack_int LAPACKE_zgesdd(int, char, lapack_int, lapack_int,
        lapack_complex_double *, lapack_int, double *,
        lapack_complex_double *, lapack_int, lapack_complex_double *,
        lapack_int);
lapack_int LAPACKE_dgesdd_work(int, char, lapack_int, lapack_int, double *,
        lapack_int, double *, double *, lapack_int, double *, lapack_int,
        double *, lapack_int, lapack_int *);
lapack_int LAPACKE_zgesdd_work(int, char, lapack_int, lapack_int,
        lapack_complex_double *, lapack_int, double *,
        lapack_complex_double *, lapack_int, lapack_complex_double *,
        lapack_int, lapack_complex_double *, lapack_int, double *,
        lapack_int *);
lapack_int LAPACKE_dgeqrf_work(int, lapack_int, lapack_int, double *,
        lapack_int, double *, double *, lapack_int);
lapack_int LAPACKE_zgeqrf_work(int, lapack_int, lapack_int,
        lapack_complex_double *, lapack_int, lapack_complex_double *,
        lapack_complex_double *, lapack_int);
lapack_int LAPACKE_dorgqr_work(int, lapack_int, lapack_int, lapack_int,
        double *, lapack_int, const double *, double *, lapack_int);
lapack_int LAPACKE_zungqr_work(int, lapack_int, lapack_int, lapack_int,
        lapack_complex_double *, lapack_int, const lapack_complex_double *,
        lapack_complex_double *, lapack_int);
lapack_int LAPACKE_dgeqp3_work(int, lapack_int, lapack_int, double *,
        lapack_int, lapack_int *, double *, double *, lapack_int);
lapack_int LAPACKE_dlarnv_work(lapack_int, lapack_int *, lapack_int,
        double *);
lapack_int LAPACKE_zlarnv_work(lapack_int, lapack_int *, lapack_int,
        lapack_complex_double *);
lapack_int LAPACKE_dpotrf(int, char, lapack_int, double *, lapack_int);
lapack_int LAPACKE_spotrf(int, char, lapack_int, float *, lapack_int);
lapack_int LAPACKE_cpotrf(int, char, lapack_int, lapack_complex_float *,
        lapack_int);
lapack_int LAPACKE_zpotrf(int, char, lapack_int, lapack_complex_double *,
        lapack_int);
#endif
