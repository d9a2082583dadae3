/* Point sets (particles) for kernel matrices.
 *
 * Layout is the reference's (include/starsh-particles.h:36-47): `count`
 * points of dimension `ndim`, stored coordinate-major ("SoA"):
 * point[d*count + i] is coordinate d of point i. */
#ifndef STARSH_B200_PARTICLES_H
#define STARSH_B200_PARTICLES_H
#include <stdio.h>
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
/* Particle files in the reference's formats (src/applications/
 * particles.c:789-1088): STARSH_ASCII, a "count=<n>, ndim=<d>" header and
 * one line per point with "%lf" coordinates separated by ", " (six
 * decimals, as the reference prints them); STARSH_BINARY, count (size_t),
 * ndim (int) and the coordinate-major doubles.  Errors as the reference:
 * STARSH_FILE_NOT_EXIST (cannot open), STARSH_FILE_WRONG_INPUT (malformed
 * or short), STARSH_FPRINTF_ERROR / STARSH_FWRITE_ERROR (write failed),
 * STARSH_WRONG_PARAMETER (unknown file type). */
int starsh_particles_read_from_file(STARSH_particles **data,
        const char *fname, const enum STARSH_FILE_TYPE ftype);
int starsh_particles_read_from_file_pointer(STARSH_particles **data,
        FILE *fp, const enum STARSH_FILE_TYPE ftype);
int starsh_particles_read_from_file_pointer_ascii(STARSH_particles **data,
        FILE *fp);
int starsh_particles_read_from_file_pointer_binary(STARSH_particles **data,
        FILE *fp);
int starsh_particles_write_to_file(const STARSH_particles *data,
        const char *fname, const enum STARSH_FILE_TYPE ftype);
int starsh_particles_write_to_file_pointer(const STARSH_particles *data,
        FILE *fp, const enum STARSH_FILE_TYPE ftype);
int starsh_particles_write_to_file_pointer_ascii(const STARSH_particles *data,
        FILE *fp);
int starsh_particles_write_to_file_pointer_binary(const STARSH_particles *data,
        FILE *fp);
/* In-place Z-order (Morton) sort; reference src/applications/
 * particles.c:1090-1221. */
int starsh_particles_zsort_inplace(STARSH_particles *data);

#ifdef __cplusplus
}
#endif
#endif
