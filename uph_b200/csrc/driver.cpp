// libuph_driver: a minimal host caller of the drop-in derivatives() (see
// include/uph_driver.h).  It owns a System laid out as the reference's
// (uph_system.h), fills it from a uph_state, and runs src/bin/sph.cc's
// leapfrog on the host, calling derivatives() of libuph_sph.so once per step.
//
// The leapfrog follows sph.cc:79-168 statement by statement (the update
// formulas and their order must be the same for the trajectory to be the
// reference's); its loops run over the particles only (sph.cc copies whole
// MaxNumberOfParticles-long arrays where entries past the particles are never
// read).  Built with -ffp-contract=off: no fused multiply-add, so every
// update rounds as the reference's does.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "uph_driver.h"

namespace {

// the System plus what the driver needs besides it; `sys` comes first so a
// System* handed out is also a pointer to its Owned
struct Owned {
  System sys;
  int itime = 0;
  std::vector<void *> blocks;  // posix_memalign
  std::vector<void *> pinned;  // cudaMallocHost
};

// The System's arrays are page-locked host memory (cudaMallocHost), so the
// drop-in's copies to and from the device go straight over the bus; plain
// host memory if page-locking is refused.
template <typename T>
T *alloc_array(Owned *o, size_t count)
{
  const size_t bytes = sizeof(T) * (count ? count : 1);
  void *p = nullptr;
  if (cudaMallocHost(&p, bytes) == cudaSuccess) {
    o->pinned.push_back(p);
  } else {
    cudaGetLastError();
    if (posix_memalign(&p, 64, bytes) != 0) throw std::bad_alloc();
    o->blocks.push_back(p);
  }
  memset(p, 0, bytes);
  return (T *)p;
}

// [rows][cols] as row pointers into one contiguous block (System.c:10-18)
double **alloc_matrix(Owned *o, size_t rows, size_t cols)
{
  double **m = alloc_array<double *>(o, rows);
  double *block = alloc_array<double>(o, rows * cols);
  for (size_t r = 0; r < rows; r++) m[r] = block + r * cols;
  return m;
}

Owned *owned(System *s) { return reinterpret_cast<Owned *>(s); }

}  // namespace

// ---- the two libSPH functions derivatives() calls back ------------------------
// (handed to the drop-in with uph_dropin_set_callbacks before every call, so
// another caller loaded into the same process cannot take their place)
namespace {

void driver_inoutflow(System *) {}

// The state effects of inputbp (src/lib/inputbp.c:192-299) for the walls of
// the resident path: boundary and solid particles carry the rest density and
// zero local pressure, and the piston (movingBoundary 1) sits at
// x = S/2 (1 - cos w t) with velocity S/2 w sin w t.  The reference also
// re-reads the boundary decks from disk here; the driver keeps them in memory.
void driver_inputbp(System *sys, double t)
{
  const int nf = sys->NumberOfFluidParticles;
  const int nw = sys->NumberOfBoundaryParticles + sys->NumberOfSolidParticles;
  for (int i = nf; i < nf + nw; i++) {
    sys->localDensity[i] = sys->density0;
    sys->localPressure[i] = 0.0;
  }
  if (sys->movingBoundary == 1 && sys->flagInitSimul == 1) {
    const double x = 0.5 * sys->stroke * (1.0 - cos(sys->omega * t));
    const double u = 0.5 * sys->stroke * sys->omega * sin(sys->omega * t);
    const int m0 = nf + sys->NumberOfSolidParticles + sys->NumberOfFixedBoundaryParticles;
    for (int i = 0; i < sys->NumberOfMovingBoundaryParticles; i++) {
      sys->Position[m0 + i][0] = x;
      sys->Velocity[m0 + i][0] = u;
      sys->localVelocity[m0 + i][0] = u;
    }
  }
}

}  // namespace

// ---- the driver ------------------------------------------------------------------

extern "C" System *uph_driver_create(const uph_params *p, const uph_state *init, int32_t max_particles)
{
  if (!p || !init || !init->Position || !init->Velocity || !init->density || !init->DynamicPressure ||
      !init->mass || !init->itype)
    return nullptr;
  const int nf = p->n_fluid, ns = p->n_solid, nb = p->n_fixed + p->n_moving;
  const int n = nf + ns + nb;
  if (n <= 0 || max_particles < n) return nullptr;
  Owned *o = new Owned();
  memset(&o->sys, 0, sizeof(System));
  System *s = &o->sys;
  // The arrays derivatives() may write past the particles -- the rate
  // arrays it zeroes and the pair list -- hold max_particles entries, as the
  // reference sizes all of them (System.c:195-260); the others hold the n
  // particles, which is all that derivatives() and the leapfrog read.
  const size_t M = (size_t)max_particles, N = (size_t)n;
  try {
    s->itype = alloc_array<int>(o, N);
    s->Position = alloc_matrix(o, N, 2);
    s->Velocity = alloc_matrix(o, N, 2);
    s->Velocity_xsph = alloc_matrix(o, N, 2);
    s->Velocity_min = alloc_matrix(o, N, 2);
    s->localVelocity = alloc_matrix(o, N, 2);
    s->velocityFluctuation = alloc_matrix(o, N, 2);
    s->dvdt = alloc_matrix(o, M, 2);
    s->dvdt_approx = alloc_matrix(o, M, 2);
    s->dwcdx = alloc_matrix(o, M, 2);
    for (double **f : {&s->mass, &s->Pressure, &s->hsml, &s->density, &s->density_min, &s->viscosity,
                       &s->DynamicPressure, &s->DynamicPressure_min, &s->densityFluctuation, &s->pressureFluctuation,
                       &s->localDensity, &s->localPressure, &s->thermalDiffusivity, &s->spongeFactor})
      *f = alloc_array<double>(o, N);
    for (double **f : {&s->ddensitydt, &s->dpdt, &s->ddensitydt_approx, &s->dpdt_approx, &s->rij2, &s->w})
      *f = alloc_array<double>(o, M);
    s->i_pair = alloc_array<int>(o, M);
    s->j_pair = alloc_array<int>(o, M);
  } catch (const std::bad_alloc &) {
    uph_driver_destroy(s);
    return nullptr;
  }
  // scalars as CreateSystem leaves them (System.c:60-335)
  s->dim = 2;
  s->MaxNumberOfParticles = max_particles;
  s->NumberOfFluidParticles = nf;
  s->NumberOfSolidParticles = ns;
  s->NumberOfFixedBoundaryParticles = p->n_fixed;
  s->NumberOfMovingBoundaryParticles = p->n_moving;
  s->NumberOfBoundaryParticles = nb;
  s->dx = p->dx;
  s->dy = p->dy;
  s->stroke = p->stroke;
  s->wavePeriod = p->wave_period;
  s->LocalDepth = p->local_depth;
  s->FlatBottomLength = p->flat_bottom_length;
  s->density0 = p->density0;
  s->AdiabaticConstant = p->adiabatic_constant;
  s->Gravity = p->gravity;
  s->viscosity0 = p->viscosity0;
  s->machNumber = p->mach_number;
  s->pecletNumber = p->peclet_number;
  s->epsilon = p->epsilon;
  s->alpha = p->alpha;
  s->virtualType = p->virtual_type;
  s->printStep = p->print_step;
  s->screenStep = p->screen_step;
  s->timeStep = p->time_step;
  s->lidVelocity = p->lid_velocity;
  s->nearNeighbor = p->near_neighbor;
  s->selectBoundaryForce = p->select_boundary_force;
  s->lennardSelect = p->lennard_select;
  s->springConstant0 = p->spring_constant0;
  s->dampingConstant0 = p->damping_constant0;
  s->flagInitSimul = p->flag_init_simul;
  s->gravityFlag = p->gravity_flag;
  s->thermalDiffusivity0 = p->thermal_diffusivity0;
  s->movingBoundary = p->moving_boundary;
  s->NumberOfInitializationSteps = p->number_of_initialization_steps;
  s->pressureProbeX = p->pressure_probe_x;
  s->pressureProbeY = p->pressure_probe_y;
  s->stressType = p->stress_type;
  s->disspationControlVolume = p->dissipation_control_volume;
  s->SpeedOfSound = p->speed_of_sound;
  s->CompressionFactor = p->compression_factor;
  s->omega = p->omega;
  s->eta = p->eta;
  s->LennardCoefficient = p->lennard_coefficient;
  s->spongeFactor0 = p->sponge_factor0;
  s->spongePosition0 = p->sponge_position0;
  s->waveAbsorption = p->wave_absorption;
  // per-particle state (input.c:105-145, inputbp.c:283-299)
  for (int i = 0; i < n; i++) {
    s->Position[i][0] = init->Position[2 * i];
    s->Position[i][1] = init->Position[2 * i + 1];
    s->Velocity[i][0] = init->Velocity[2 * i];
    s->Velocity[i][1] = init->Velocity[2 * i + 1];
    const double *lv = init->localVelocity ? init->localVelocity : init->Velocity;
    s->localVelocity[i][0] = lv[2 * i];
    s->localVelocity[i][1] = lv[2 * i + 1];
    s->density[i] = init->density[i];
    s->localDensity[i] = init->localDensity ? init->localDensity[i] : init->density[i];
    s->DynamicPressure[i] = init->DynamicPressure[i];
    s->localPressure[i] = init->localPressure ? init->localPressure[i] : 0.0;
    s->mass[i] = init->mass[i];
    s->itype[i] = init->itype[i];
    s->hsml[i] = p->h;
    s->viscosity[i] = p->viscosity0;
    s->thermalDiffusivity[i] = p->thermal_diffusivity0;
  }
  if (init->spongeFactor)
    for (int i = 0; i < nf; i++) s->spongeFactor[i] = init->spongeFactor[i];
  // sph.cc:79-87
  memcpy(s->density_min, s->density, sizeof(double) * nf);
  memcpy(s->DynamicPressure_min, s->DynamicPressure, sizeof(double) * nf);
  return s;
}

extern "C" uph_status uph_driver_step(System *sys, int32_t nsteps)
{
  if (!sys || nsteps < 0) return UPH_BAD_ARG;
  Owned *o = owned(sys);
  const int nf = sys->NumberOfFluidParticles;
  const int n = nf + sys->NumberOfSolidParticles + sys->NumberOfBoundaryParticles;
  const double dt = sys->timeStep;
  double *const rho = sys->density, *const rhot = sys->localDensity, *const p = sys->DynamicPressure;
  double *const pt = sys->localPressure, *const rho_min = sys->density_min, *const p_min = sys->DynamicPressure_min;
  for (int k = 0; k < nsteps; k++) {
    const int itime = ++o->itime;
    const double t = itime * dt;
    if (itime != 1) {
      // sph.cc:93-124; its copies (sph.cc:94-99) done inside the parallel
      // loop, element by element: the walls' velocity copies first
#pragma omp parallel for schedule(static)
      for (int i = nf; i < n; i++)
        for (int d = 0; d < 2; d++) {
          sys->localVelocity[i][d] = sys->Velocity[i][d];
          sys->Velocity_min[i][d] = sys->Velocity[i][d];
        }
#pragma omp parallel for schedule(static)
      for (int i = 0; i < nf; i++) {
        rho_min[i] = rho[i];
        p_min[i] = p[i];
        rhot[i] = rho[i];
        pt[i] = p[i];
        for (int d = 0; d < 2; d++) sys->localVelocity[i][d] = sys->Velocity[i][d];
        rho[i] += 0.5 * dt * sys->ddensitydt_approx[i];
        rhot[i] = rhot[i] + 0.5 * dt * sys->ddensitydt_approx[i] + sys->densityFluctuation[i];
        p[i] += 0.5 * dt * sys->dpdt_approx[i];
        pt[i] = pt[i] + 0.5 * dt * sys->dpdt_approx[i] + sys->pressureFluctuation[i];
        for (int d = 0; d < 2; d++) {
          sys->Velocity_min[i][d] = sys->Velocity[i][d];
          sys->Velocity_xsph[i][d] += 0.5 * dt * sys->dvdt[i][d];
          sys->Velocity[i][d] += 0.5 * dt * sys->dvdt_approx[i][d];
          sys->localVelocity[i][d] =
              sys->Velocity[i][d] + 0.5 * dt * sys->dvdt_approx[i][d] + sys->epsilon * sys->velocityFluctuation[i][d];
        }
      }
    } else {
      memcpy(sys->Velocity_xsph[0], sys->Velocity[0], sizeof(double) * 2 * n);
    }
    uph_dropin_set_callbacks(driver_inputbp, driver_inoutflow);
    derivatives(sys, t);
    if (itime == 1) {
      // sph.cc:131-146
#pragma omp parallel for schedule(static)
      for (int i = 0; i < nf; i++) {
        rhot[i] = rho[i] + 0.5 * dt * sys->ddensitydt[i] + sys->densityFluctuation[i];
        rho[i] += 0.5 * dt * sys->ddensitydt[i];
        pt[i] = p[i] + 0.5 * dt * sys->dpdt[i] + sys->pressureFluctuation[i];
        p[i] += 0.5 * dt * sys->dpdt[i];
        for (int d = 0; d < 2; d++) {
          sys->Velocity_xsph[i][d] =
              sys->Velocity[i][d] + 0.5 * dt * sys->dvdt[i][d] + sys->epsilon * sys->velocityFluctuation[i][d];
          sys->localVelocity[i][d] =
              sys->Velocity[i][d] + 0.5 * dt * sys->dvdt[i][d] + sys->epsilon * sys->velocityFluctuation[i][d];
          sys->Velocity[i][d] += 0.5 * dt * sys->dvdt[i][d];
          sys->Position[i][d] += dt * sys->Velocity[i][d];
        }
      }
    } else {
      // sph.cc:147-162
#pragma omp parallel for schedule(static)
      for (int i = 0; i < nf; i++) {
        rhot[i] = rho_min[i] + dt * sys->ddensitydt[i] + sys->densityFluctuation[i];
        rho[i] = rho_min[i] + dt * sys->ddensitydt[i];
        pt[i] = p_min[i] + dt * sys->dpdt[i] + sys->pressureFluctuation[i];
        p[i] = p_min[i] + dt * sys->dpdt[i];
        for (int d = 0; d < 2; d++) {
          sys->Velocity_xsph[i][d] =
              sys->Velocity_min[i][d] + dt * sys->dvdt[i][d] + sys->epsilon * sys->velocityFluctuation[i][d];
          sys->localVelocity[i][d] =
              sys->Velocity_min[i][d] + dt * sys->dvdt[i][d] + sys->epsilon * sys->velocityFluctuation[i][d];
          sys->Velocity[i][d] = sys->Velocity_min[i][d] + dt * sys->dvdt[i][d];
          sys->Position[i][d] += dt * sys->Velocity[i][d];
        }
      }
    }
  }
  return UPH_OK;
}

extern "C" uph_status uph_driver_state(const System *sys, uph_state *out)
{
  if (!sys || !out) return UPH_BAD_ARG;
  const int nf = sys->NumberOfFluidParticles;
  const int n = nf + sys->NumberOfSolidParticles + sys->NumberOfBoundaryParticles;
  auto copy = [](double *dst, const double *src, size_t count) {
    if (dst) memcpy(dst, src, sizeof(double) * count);
  };
  copy(out->Position, sys->Position[0], 2 * (size_t)n);
  copy(out->Velocity, sys->Velocity[0], 2 * (size_t)n);
  copy(out->localVelocity, sys->localVelocity[0], 2 * (size_t)n);
  copy(out->density, sys->density, n);
  copy(out->localDensity, sys->localDensity, n);
  copy(out->DynamicPressure, sys->DynamicPressure, n);
  copy(out->localPressure, sys->localPressure, n);
  copy(out->mass, sys->mass, n);
  if (out->itype) memcpy(out->itype, sys->itype, sizeof(int) * n);
  copy(out->Velocity_min, sys->Velocity_min[0], 2 * (size_t)nf);
  copy(out->density_min, sys->density_min, nf);
  copy(out->DynamicPressure_min, sys->DynamicPressure_min, nf);
  copy(out->spongeFactor, sys->spongeFactor, nf);
  copy(out->ddensitydt, sys->ddensitydt, nf);
  copy(out->dpdt, sys->dpdt, nf);
  copy(out->dvdt, sys->dvdt[0], 2 * (size_t)nf);
  copy(out->ddensitydt_approx, sys->ddensitydt_approx, nf);
  copy(out->dpdt_approx, sys->dpdt_approx, nf);
  copy(out->dvdt_approx, sys->dvdt_approx[0], 2 * (size_t)nf);
  copy(out->densityFluctuation, sys->densityFluctuation, nf);
  copy(out->pressureFluctuation, sys->pressureFluctuation, nf);
  copy(out->velocityFluctuation, sys->velocityFluctuation[0], 2 * (size_t)nf);
  copy(out->Pressure, sys->Pressure, n);
  return UPH_OK;
}

extern "C" void uph_driver_destroy(System *sys)
{
  if (!sys) return;
  Owned *o = owned(sys);
  for (void *b : o->blocks) free(b);
  for (void *b : o->pinned) cudaFreeHost(b);
  delete o;
}
