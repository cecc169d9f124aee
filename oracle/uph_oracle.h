/*
 * Test infrastructure (oracle only): CPU restatement of the reference's
 * per-timestep hot path, used by the tests, by smoke() and by bench.py's CPU
 * baseline as the checker of the CUDA library.  The product never links it.
 */
#ifndef UPH_ORACLE_H
#define UPH_ORACLE_H

#include <stdint.h>
#include "../include/uph.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct uph_oracle uph_oracle;

uph_oracle *uph_oracle_create(const uph_params *p);
void uph_oracle_destroy(uph_oracle *o);
int uph_oracle_set_state(uph_oracle *o, const uph_state *st, int itime);
int uph_oracle_get_state(const uph_oracle *o, uph_state *st);
/* one rate evaluation at time t (REF: derivatives.c:3137-4327 hot path;
   WCSPH: the textbook profile) */
int uph_oracle_derivatives(uph_oracle *o, double t);
/* nsteps of the sph.cc:90-168 leapfrog */
int uph_oracle_step(uph_oracle *o, int nsteps);
int64_t uph_oracle_pairs(const uph_oracle *o, int64_t cap, int32_t *i_pair, int32_t *j_pair, double *rij2,
                         double *w, double *dwcdx);
int uph_oracle_max_neighbors(const uph_oracle *o);
/* per-particle shaking of the moving block (NULL: the movingBoundary mode) */
void uph_oracle_set_wall_motion(uph_oracle *o, const double *x0, const double *hs, const double *om);
void uph_oracle_energies(const uph_oracle *o, double out[3]);

/* stand-alone radius search with SearchNeighbors' filter (Search.cc:31-40) */
int64_t uph_oracle_search(const double *pos, int n_fluid, int n_all, int particle_boundary, double dist, int64_t cap,
                          int32_t *i_pair, int32_t *j_pair, double *rij2, int *max_inradius);

#ifdef __cplusplus
}
#endif
#endif
