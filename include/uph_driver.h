/*
 * uph_driver.h -- a host caller of the drop-in derivatives().
 *
 * The reference's own caller is a program, src/bin/sph.cc, linked against
 * the rest of libSPH (CreateSystem, input, inputbp, output).  libuph_driver.so
 * is a minimal stand-in for that caller, for applications and benchmarks
 * without a libSPH: it allocates a System with the reference's layout
 * (uph_system.h), fills it from a uph_state, and runs sph.cc's leapfrog
 * (src/bin/sph.cc:79-168) on the host around the drop-in derivatives() of
 * libuph_sph.so -- every step crosses the host/device boundary the way a
 * relinked reference does.  It also provides the two libSPH functions
 * derivatives() calls back (inputbp, inoutflow) for the fixed walls and the
 * piston of the resident path; it is not meant to be linked together with
 * the reference's own libSPH.  No counterpart in the reference as a library.
 */
#ifndef UPH_DRIVER_H
#define UPH_DRIVER_H

#include "uph.h"
#include "uph_system.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A System for p's counts with MaxNumberOfParticles = max_particles (>= all
 * particles): the pair arrays and the rate arrays derivatives() zeroes hold
 * max_particles entries, the other per-particle arrays the particles; all
 * in page-locked host memory when the driver grants it.  Filled from `init`
 * (Position, Velocity, density,
 * DynamicPressure, mass and itype required; localVelocity / localDensity /
 * localPressure default to the plain fields).  NULL on bad arguments or
 * when host memory runs out. */
System *uph_driver_create(const uph_params *p, const uph_state *init, int32_t max_particles);

/* nsteps leapfrog steps of src/bin/sph.cc:90-168, each with one
 * derivatives(sys, t) call; the step counter continues across calls. */
uph_status uph_driver_step(System *sys, int32_t nsteps);

/* Copies the System's fields into `out` (any member may be NULL). */
uph_status uph_driver_state(const System *sys, uph_state *out);

void uph_driver_destroy(System *sys);

#ifdef __cplusplus
}
#endif

#endif /* UPH_DRIVER_H */
