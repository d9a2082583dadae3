/* Electrodynamics problem: Helmholtz kernels sin(k r)/r and cos(k r)/r,
 * r = 0 giving `diag` (reference: include/starsh-electrodynamics.h:34-79). */
#ifndef STARSH_B200_ELECTRODYNAMICS_H
#define STARSH_B200_ELECTRODYNAMICS_H
#include "starsh.h"
#include "starsh-particles.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct starsh_eddata
{
    STARSH_particles particles;
    double k;
    double diag;
} STARSH_eddata;

enum STARSH_ELECTRODYNAMICS_KERNEL
{
    STARSH_ELECTRODYNAMICS_SIN = 1,
    STARSH_ELECTRODYNAMICS_COS = 2,
    STARSH_ELECTRODYNAMICS_SIN_SIMD = 11,
    STARSH_ELECTRODYNAMICS_COS_SIMD = 12,
};

enum STARSH_ELECTRODYNAMICS_PARAM
{
    STARSH_ELECTRODYNAMICS_NDIM = 1,
    STARSH_ELECTRODYNAMICS_K = 2,
    STARSH_ELECTRODYNAMICS_DIAG = 3,
    STARSH_ELECTRODYNAMICS_PLACE = 4,
};

int starsh_eddata_init(STARSH_eddata **data, STARSH_int count, int ndim,
        double *point, double k, double diag);
int starsh_eddata_generate(STARSH_eddata **data, STARSH_int count, int ndim,
        double k, double diag, enum STARSH_PARTICLES_PLACEMENT place);
int starsh_eddata_generate_va(STARSH_eddata **data, STARSH_int count,
        va_list args);
int starsh_eddata_generate_el(STARSH_eddata **data, STARSH_int count, ...);
int starsh_eddata_get_kernel(STARSH_kernel **kernel, STARSH_eddata *data,
        enum STARSH_ELECTRODYNAMICS_KERNEL type);
void starsh_eddata_free(STARSH_eddata *data);

#define STARSH_B200_DECLARE_ED(fam) \
    STARSH_kernel starsh_eddata_block_##fam##_kernel_1d, \
        starsh_eddata_block_##fam##_kernel_2d, \
        starsh_eddata_block_##fam##_kernel_3d, \
        starsh_eddata_block_##fam##_kernel_4d, \
        starsh_eddata_block_##fam##_kernel_nd, \
        starsh_eddata_block_##fam##_kernel_1d_simd, \
        starsh_eddata_block_##fam##_kernel_2d_simd, \
        starsh_eddata_block_##fam##_kernel_3d_simd, \
        starsh_eddata_block_##fam##_kernel_4d_simd, \
        starsh_eddata_block_##fam##_kernel_nd_simd;
STARSH_B200_DECLARE_ED(sin)
STARSH_B200_DECLARE_ED(cos)

#ifdef __cplusplus
}
#endif
#endif
