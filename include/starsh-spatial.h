/* Spatial statistics problem: covariance kernels of a Gaussian process.
 *
 * STARSH_ssdata layout and parameter enums as in the reference
 * (include/starsh-spatial.h:35-179).  `sigma` is used directly as the
 * variance (sigma^2 in the formulas). */
#ifndef STARSH_B200_SPATIAL_H
#define STARSH_B200_SPATIAL_H
#include "starsh.h"
#include "starsh-particles.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct starsh_ssdata
{
    STARSH_particles particles;
    double beta;
    double nu;
    double noise;
    double sigma;
    double nu2;
    double sigma2;
    double corr;
} STARSH_ssdata;

enum STARSH_SPATIAL_KERNEL
{
    STARSH_SPATIAL_EXP = 1,
    STARSH_SPATIAL_SQREXP = 2,
    STARSH_SPATIAL_MATERN = 3,
    STARSH_SPATIAL_MATERN2 = 4,
    STARSH_SPATIAL_EXP_SIMD = 11,
    STARSH_SPATIAL_SQREXP_SIMD = 12,
    STARSH_SPATIAL_MATERN_SIMD = 13,
    STARSH_SPATIAL_MATERN2_SIMD = 14,
};

enum STARSH_SPATIAL_PARAM
{
    STARSH_SPATIAL_NDIM = 1,
    STARSH_SPATIAL_BETA = 2,
    STARSH_SPATIAL_NU = 3,
    STARSH_SPATIAL_NOISE = 4,
    STARSH_SPATIAL_PLACE = 5,
    STARSH_SPATIAL_SIGMA = 6,
    STARSH_SPATIAL_SIGMA2 = 7,
    STARSH_SPATIAL_NU2 = 8,
    STARSH_SPATIAL_CORR = 9,
};

int starsh_ssdata_new(STARSH_ssdata **data, STARSH_int count, int ndim);
int starsh_ssdata_init(STARSH_ssdata **data, STARSH_int count, int ndim,
        double *point, double beta, double nu, double noise, double sigma);
int starsh_ssdata_generate(STARSH_ssdata **data, STARSH_int count, int ndim,
        double beta, double nu, double noise,
        enum STARSH_PARTICLES_PLACEMENT place, double sigma);
int starsh_ssdata_generate_va(STARSH_ssdata **data, STARSH_int count,
        va_list args);
int starsh_ssdata_generate_el(STARSH_ssdata **data, STARSH_int count, ...);
int starsh_ssdata_get_kernel(STARSH_kernel **kernel, STARSH_ssdata *data,
        enum STARSH_SPATIAL_KERNEL type);
void starsh_ssdata_free(STARSH_ssdata *data);

/* Kernel entry points.  In this library each one evaluates the block on the
 * GPU and copies it to `result` (host memory); the approximation engine
 * recognises these functions and generates tiles on the device instead of
 * calling them.  Formulas: exp sigma*exp(-r/beta); sqexp
 * sigma*exp(-r^2/(2 beta^2)); Matern sigma*2^(1-nu)/Gamma(nu)*x^nu*K_nu(x)
 * with x = r*sqrt(2 nu)/beta (Matern2: x = r/beta); r = 0 gives
 * sigma+noise (reference: src/applications/spatial/kernel_*.c). */
#define STARSH_B200_DECLARE_SPATIAL(fam) \
    STARSH_kernel starsh_ssdata_block_##fam##_kernel_1d, \
        starsh_ssdata_block_##fam##_kernel_2d, \
        starsh_ssdata_block_##fam##_kernel_3d, \
        starsh_ssdata_block_##fam##_kernel_4d, \
        starsh_ssdata_block_##fam##_kernel_nd, \
        starsh_ssdata_block_##fam##_kernel_1d_simd, \
        starsh_ssdata_block_##fam##_kernel_2d_simd, \
        starsh_ssdata_block_##fam##_kernel_3d_simd, \
        starsh_ssdata_block_##fam##_kernel_4d_simd, \
        starsh_ssdata_block_##fam##_kernel_nd_simd;
STARSH_B200_DECLARE_SPATIAL(exp)
STARSH_B200_DECLARE_SPATIAL(sqrexp)
STARSH_B200_DECLARE_SPATIAL(matern)
STARSH_B200_DECLARE_SPATIAL(matern2)

#ifdef __cplusplus
}
#endif
#endif
