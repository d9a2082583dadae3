/* RBF (mesh deformation) problem: radial basis functions phi(|x_i-x_j|/rad)
 * on 3-D points stored point-major ("AoS"): mesh[3*i + d]
 * (reference: include/starsh-rbf.h:29-63, src/applications/
 * mesh_deformation/virus.c:41-94, cube.c:37-83).  kernel: 0 Gaussian
 * exp(-x^2), 1 exp(-x), 2 1/(1+x^2), 3 1/sqrt(1+x^2), 4 and 5 exp(-x)+(1+x),
 * 6 x^2 log x, 7 (1-x)^5 for x<=1, 8 1+x^2, otherwise Wendland
 * (1-x)^4 (4x+1) for x<=1.  `reg` is added on the diagonal when `isreg`. */
#ifndef STARSH_B200_RBF_H
#define STARSH_B200_RBF_H
#include "starsh.h"
#include "starsh-particles.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct starsh_mddata
{
    STARSH_particles particles;
    double reg;
    int kernel;
    int numobj;
    int isreg;
    double rad;
    double denst;
    int mesh_points;
    int mordering;
} STARSH_mddata;

/* Builds an STARSH_mddata over caller-owned AoS coordinates (3*count
 * doubles).  B200 addition: the reference only builds mddata from mesh
 * files (src/applications/mesh_deformation/mesh_rbf.c:219-334). */
int starsh_mddata_init(STARSH_mddata **data, STARSH_int count, double *mesh,
        int kernel, int numobj, int isreg, double reg, double rad,
        double denst);
void starsh_mddata_free(STARSH_mddata *data);

STARSH_kernel starsh_generate_3d_virus, starsh_generate_3d_cube;

#ifdef __cplusplus
}
#endif
#endif
