/* Point sets (particles) for kernel matrices.
 *
 * Layout is the reference's (include/starsh-particles.h:36-47): `count`
 * points of dimension `ndim`, stored coordinate-major ("SoA"):
 * point[d*count + i] is coordinate d of point i. */
#ifndef STARSH_B200_PARTICLES_H
#define STARSH_B200_PARTICLES_H
#include "starsh.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct starsh_particles
{
    STARSH_int count;
    int ndim;
    double *point;
} STARSH_particles;

/* Placement strategies; values as in the reference
 * (include/starsh-particles.h:50-67).  The B200 library generates RAND,
 * UNIFORM and QUASIUNIFORM1 (the placements the approximation tests use);
 * the others return STARSH_WRONG_PARAMETER. */
enum STARSH_PARTICLES_PLACEMENT
{
    STARSH_PARTICLES_RAND = 1,
    STARSH_PARTICLES_UNIFORM = 3,
    STARSH_PARTICLES_RANDGRID = 4,
    STARSH_PARTICLES_QUASIUNIFORM1 = 6,
    STARSH_PARTICLES_QUASIUNIFORM2 = 7,
    STARSH_PARTICLES_OBSOLETE1 = -1,
    STARSH_PARTICLES_OBSOLETE2 = -2,
    STARSH_PARTICLES_OBSOLETE3 = -3,
    STARSH_PARTICLES_OBSOLETE4 = -4,
};

int starsh_particles_new(STARSH_particles **data, STARSH_int count, int ndim);
int starsh_particles_init(STARSH_particles **data, STARSH_int count, int ndim,
        double *point);
void starsh_particles_free(STARSH_particles *data);
int starsh_particles_generate(STARSH_particles **data, STARSH_int count,
        int ndim, enum STARSH_PARTICLES_PLACEMENT ptype);
int starsh_particles_generate_rand(STARSH_particles **data, STARSH_int count,
        int ndim);
int starsh_particles_generate_uniform(STARSH_particles **data,
        STARSH_int count, int ndim);
int starsh_particles_generate_quasiuniform1(STARSH_particles **data,
        STARSH_int count, int ndim);
/* In-place Z-order (Morton) sort; reference src/applications/
 * particles.c:1090-1221. */
int starsh_particles_zsort_inplace(STARSH_particles *data);

#ifdef __cplusplus
}
#endif
#endif
