/* Electrostatics problem: Coulomb potential 1/r between particles
 * (reference: include/starsh-electrostatics.h:35-50).  r = 0 gives 0, as in
 * the reference; a regularised diagonal is available through
 * starsh_b200_kernel_register() (starsh-b200.h). */
#ifndef STARSH_B200_ELECTROSTATICS_H
#define STARSH_B200_ELECTROSTATICS_H
#include "starsh.h"
#include "starsh-particles.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef STARSH_particles STARSH_esdata;

enum STARSH_ELECTROSTATICS_KERNEL
{
    STARSH_ELECTROSTATICS_COULOMB_POTENTIAL = 1,
    STARSH_ELECTROSTATICS_COULOMB_POTENTIAL_SIMD = 2,
};

enum STARSH_ELECTROSTATICS_PARAM
{
    STARSH_ELECTROSTATICS_NDIM = 1,
    STARSH_ELECTROSTATICS_PLACE = 2,
};

int starsh_esdata_init(STARSH_esdata **data, STARSH_int count, int ndim,
        double *point);
int starsh_esdata_generate(STARSH_esdata **data, STARSH_int count, int ndim,
        enum STARSH_PARTICLES_PLACEMENT place);
int starsh_esdata_generate_va(STARSH_esdata **data, STARSH_int count,
        va_list args);
int starsh_esdata_generate_el(STARSH_esdata **data, STARSH_int count, ...);
int starsh_esdata_get_kernel(STARSH_kernel **kernel, STARSH_esdata *data,
        enum STARSH_ELECTROSTATICS_KERNEL type);
void starsh_esdata_free(STARSH_esdata *data);

STARSH_kernel starsh_esdata_block_coulomb_potential_kernel_1d,
    starsh_esdata_block_coulomb_potential_kernel_2d,
    starsh_esdata_block_coulomb_potential_kernel_3d,
    starsh_esdata_block_coulomb_potential_kernel_4d,
    starsh_esdata_block_coulomb_potential_kernel_nd,
    starsh_esdata_block_coulomb_potential_kernel_1d_simd,
    starsh_esdata_block_coulomb_potential_kernel_2d_simd,
    starsh_esdata_block_coulomb_potential_kernel_3d_simd,
    starsh_esdata_block_coulomb_potential_kernel_4d_simd,
    starsh_esdata_block_coulomb_potential_kernel_nd_simd;

#ifdef __cplusplus
}
#endif
#endif
