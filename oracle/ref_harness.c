/*
 * Test infrastructure (oracle only): drives the reference's own compiled
 * solver so tests and the CPU baseline can read its state after any number
 * of steps.  Nothing in the product links this file.
 *
 * It links against the reference's unmodified sources (compiled by
 * oracle/Makefile from the reference tree): CreateSystem / input / inputbp /
 * inoutflow / output / derivatives.  What this file adds:
 *
 *   - ref_open(): the set-up of src/bin/sph.cc:23-87 -- CreateSystem, input,
 *     then zeroing the rates and copying density / DynamicPressure into their
 *     *_min arrays (sph.cc:79-87).  Two documented deviations, neither of
 *     which changes any arithmetic:
 *       * `eta_override` > 0 replaces sys->eta after CreateSystem (the decks
 *         store nearNeighbor as an int, System.c:311, so h = 1.3 dx cannot be
 *         expressed in parameters.dat; input.c:107 and inputbp.c:287 read
 *         sys->eta afterwards);
 *       * `fluid_capacity_pct` > 0 shrinks the reference's particle capacity
 *         MaxNumberOfParticles = Ns + Nb + 100 Nf + Nfr (System.c:195) to
 *         Ns + Nb + pct/100 Nf + Nfr by letting CreateSystem read a fluid
 *         count of ceil(pct/100 Nf) from a scratch directory; input() then
 *         reads the real deck.  At 100 Nf a 500k-particle deck needs
 *         ~80 GB of per-step memsets and scratch.  The pair arrays are sized
 *         by the same capacity, so the search stand-in is told the capacity
 *         and aborts instead of overflowing.
 *   - ref_step(): the leapfrog time loop of src/bin/sph.cc:90-168, restated
 *     statement by statement (same operation order, same expressions), with
 *     the per-printStep output (sph.cc:169-191) left out.
 *   - getters that copy fluid / pair arrays out.
 *
 * The reference reads its decks from the current directory (System.c:41-46,
 * input.c:28-30, inputbp.c:18-23, every step); every entry point here
 * changes into the deck directory and restores the caller's directory.
 */
#define _GNU_SOURCE
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>
#include <omp.h>

#include "System.h"
#include "derivatives.h"
#include "input.h"
#include "inputbp.h"
#include "inoutflow.h"

/* defined by shim/search_standin.c; absent when the hot path is the GPU drop-in */
extern void uph_standin_set_capacity(long cap) __attribute__((weak));
/* the drop-in build (libuph_dropin.so) hands derivatives() the reference's
 * own inputbp / inoutflow before every call, so another caller of the
 * drop-in loaded into the same process cannot take their place */
extern void uph_dropin_set_callbacks(void (*)(System *, double), void (*)(System *)) __attribute__((weak));
static void use_reference_callbacks(void)
{
  if (uph_dropin_set_callbacks) uph_dropin_set_callbacks(inputbp, inoutflow);
}

typedef struct {
  System *sys;
  char deck[4096];
  int itime;
} ref_run;

static int read_count(const char *dir, const char *name, int *out)
{
  char path[8192];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE *f = fopen(path, "r");
  if (!f) return -1;
  int ok = fscanf(f, "%d", out) == 1;
  fclose(f);
  return ok ? 0 : -1;
}

static int write_text(const char *dir, const char *name, const char *text)
{
  char path[8192];
  snprintf(path, sizeof path, "%s/%s", dir, name);
  FILE *f = fopen(path, "w");
  if (!f) return -1;
  fputs(text, f);
  fclose(f);
  return 0;
}

static int copy_file(const char *src_dir, const char *dst_dir, const char *name)
{
  char src[8192], dst[8192];
  snprintf(src, sizeof src, "%s/%s", src_dir, name);
  snprintf(dst, sizeof dst, "%s/%s", dst_dir, name);
  FILE *a = fopen(src, "rb");
  if (!a) return -1;
  FILE *b = fopen(dst, "wb");
  if (!b) { fclose(a); return -1; }
  char buf[65536];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, a)) > 0) fwrite(buf, 1, n, b);
  fclose(a);
  fclose(b);
  return 0;
}

/* Returns NULL on a missing deck file (the reference itself would exit). */
/* The reference's per-thread scratch has 64 rows (System.c:209,
 * CreateMatrix(64, ...)), indexed by omp_get_thread_num() in every pair loop
 * (derivatives.c:1741 and its siblings): a larger team writes past it. */
enum { kRefMaxThreads = 64 };

int ref_threads(void) { return omp_get_max_threads(); }

ref_run *ref_open(const char *deck_dir, double eta_override, int fluid_capacity_pct)
{
  if (omp_get_max_threads() > kRefMaxThreads) omp_set_num_threads(kRefMaxThreads);
  char cwd[8192];
  if (!getcwd(cwd, sizeof cwd)) return NULL;
  ref_run *run = (ref_run *)calloc(1, sizeof(ref_run));
  if (!realpath(deck_dir, run->deck)) { free(run); return NULL; }

  char scratch[] = "/tmp/uph_ref_capXXXXXX";
  int use_scratch = fluid_capacity_pct > 0;
  if (use_scratch) {
    int nf, nfix, nmov, nsol, nfro = 0;
    if (read_count(run->deck, "FluidParticle.dat", &nf) || read_count(run->deck, "FixedBoundaryParticle.dat", &nfix) ||
        read_count(run->deck, "MovingBoundaryParticle.dat", &nmov) || read_count(run->deck, "SolidParticle.dat", &nsol)) {
      free(run);
      return NULL;
    }
    read_count(run->deck, "FrozenParticle.dat", &nfro);
    if (!mkdtemp(scratch)) { free(run); return NULL; }
    char line[64];
    long nf_cap = ((long)nf * fluid_capacity_pct + 99) / 100;
    snprintf(line, sizeof line, "%ld\n", nf_cap);
    write_text(scratch, "FluidParticle.dat", line);
    snprintf(line, sizeof line, "%d\n", nfix);
    write_text(scratch, "FixedBoundaryParticle.dat", line);
    snprintf(line, sizeof line, "%d\n", nmov);
    write_text(scratch, "MovingBoundaryParticle.dat", line);
    snprintf(line, sizeof line, "%d\n", nsol);
    write_text(scratch, "SolidParticle.dat", line);
    snprintf(line, sizeof line, "%d\n", nfro);
    write_text(scratch, "FrozenParticle.dat", line);
    if (copy_file(run->deck, scratch, "parameters.dat")) { free(run); return NULL; }
    if (chdir(scratch)) { free(run); return NULL; }
  } else if (chdir(run->deck)) {
    free(run);
    return NULL;
  }

  System *sys = CreateSystem(128, 128); /* sph.cc:23 */
  /* CreateSystem leaves inflowParticles unset, and the first derivatives()
   * call with t > 0 runs inoutflow (derivatives.c:3162-3164), which walks
   * i_inflow[0, inflowParticles) before the inflow scan (:3172) first sets
   * the count: with whatever the heap held there it read arbitrary
   * Position rows and crashed now and then.  Zero, as the scan would leave it
   * for a deck with no inflow. */
  sys->inflowParticles = 0;
  if (use_scratch) {
    const char *names[] = {"FluidParticle.dat", "FixedBoundaryParticle.dat", "MovingBoundaryParticle.dat",
                           "SolidParticle.dat", "FrozenParticle.dat", "parameters.dat"};
    for (int k = 0; k < 6; k++) {
      char p[8192];
      snprintf(p, sizeof p, "%s/%s", scratch, names[k]);
      unlink(p);
    }
    if (chdir(run->deck)) { free(run); return NULL; }
    rmdir(scratch);
  }
  if (eta_override > 0.0) sys->eta = eta_override;
  input(sys); /* sph.cc:52 */

  /* sph.cc:79-87 */
  memset(sys->dvdt[0], 0, sizeof(double) * sys->MaxNumberOfParticles * sys->dim);
  memset(sys->ddensitydt, 0, sizeof(double) * sys->MaxNumberOfParticles);
  memcpy(sys->density_min, sys->density, sizeof(double) * sys->NumberOfFluidParticles);
  memset(sys->dpdt, 0, sizeof(double) * sys->MaxNumberOfParticles);
  memcpy(sys->DynamicPressure_min, sys->DynamicPressure, sizeof(double) * sys->NumberOfFluidParticles);
  memset(sys->dvdt_approx[0], 0, sizeof(double) * sys->MaxNumberOfParticles * sys->dim);
  memset(sys->ddensitydt_approx, 0, sizeof(double) * sys->MaxNumberOfParticles);
  memset(sys->dpdt_approx, 0, sizeof(double) * sys->MaxNumberOfParticles);

  if (uph_standin_set_capacity) uph_standin_set_capacity(sys->MaxNumberOfParticles);
  run->sys = sys;
  run->itime = 0;
  if (chdir(cwd)) { /* keep going: the run itself is valid */ }
  return run;
}

void ref_close(ref_run *run)
{
  if (!run) return;
  if (run->sys) DestroySystem(run->sys);
  free(run);
}

/* One call of the reference's derivatives() at time t, no integration. */
int ref_derivatives(ref_run *run, double t)
{
  char cwd[8192];
  if (!getcwd(cwd, sizeof cwd) || chdir(run->deck)) return -1;
  use_reference_callbacks();
  derivatives(run->sys, t);
  if (chdir(cwd)) return -1;
  return 0;
}

/* Seconds of `ncalls` calls of the reference's inputbp() at the next step's
 * time -- the per-step re-read of the boundary decks (inputbp.c:28-191) plus
 * the wall-motion law that derivatives() runs first (derivatives.c:3168).
 * Calling it again at the same time changes nothing the next step sees. */
double ref_time_inputbp(ref_run *run, int ncalls)
{
  char cwd[8192];
  if (!getcwd(cwd, sizeof cwd) || chdir(run->deck)) return -1.0;
  const double t = (run->itime + 1) * run->sys->timeStep;
  struct timespec a, b;
  clock_gettime(CLOCK_MONOTONIC, &a);
  for (int k = 0; k < ncalls; k++) inputbp(run->sys, t);
  clock_gettime(CLOCK_MONOTONIC, &b);
  if (chdir(cwd)) return -1.0;
  return (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
}

/* The time loop of src/bin/sph.cc:90-168 for `nsteps` more steps. */
int ref_step(ref_run *run, int nsteps)
{
  char cwd[8192];
  if (!getcwd(cwd, sizeof cwd) || chdir(run->deck)) return -1;
  System *sys = run->sys;
  const double dt = sys->timeStep; /* sph.cc:24 */
  for (int s = 0; s < nsteps; s++) {
    const int itime = ++run->itime;
    const double t = itime * dt;
    if (itime != 1) {
      memcpy(sys->density_min, sys->density, sizeof(double) * sys->NumberOfFluidParticles);
      memcpy(sys->DynamicPressure_min, sys->DynamicPressure, sizeof(double) * sys->NumberOfFluidParticles);
      memcpy(sys->localDensity, sys->density, sizeof(double) * sys->NumberOfFluidParticles);
      memcpy(sys->localPressure, sys->DynamicPressure, sizeof(double) * sys->NumberOfFluidParticles);
      memcpy(sys->localVelocity[0], sys->Velocity[0], sizeof(double) * sys->dim * sys->MaxNumberOfParticles);
      memcpy(sys->Velocity_min[0], sys->Velocity[0], sizeof(double) * sys->dim * sys->MaxNumberOfParticles);
      for (int i = 0; i < sys->NumberOfFluidParticles; i++) {
        sys->density[i] += 0.5 * dt * sys->ddensitydt_approx[i];
        sys->localDensity[i] = sys->localDensity[i] + 0.5 * dt * sys->ddensitydt_approx[i] + sys->densityFluctuation[i];
        sys->DynamicPressure[i] += 0.5 * dt * sys->dpdt_approx[i];
        sys->localPressure[i] = sys->localPressure[i] + 0.5 * dt * sys->dpdt_approx[i] + sys->pressureFluctuation[i];
      }
      for (int i = 0; i < sys->NumberOfFluidParticles; i++) {
        for (int d = 0; d < sys->dim; d++) {
          sys->Velocity_min[i][d] = sys->Velocity[i][d];
          sys->Velocity_xsph[i][d] += 0.5 * dt * sys->dvdt[i][d];
          sys->Velocity[i][d] += 0.5 * dt * sys->dvdt_approx[i][d];
          sys->localVelocity[i][d] = sys->Velocity[i][d] + 0.5 * dt * sys->dvdt_approx[i][d] +
                                     sys->epsilon * sys->velocityFluctuation[i][d];
        }
      }
    }
    if (itime == 1)
      memcpy(sys->Velocity_xsph[0], sys->Velocity[0], sizeof(double) * sys->dim * sys->MaxNumberOfParticles);

    use_reference_callbacks();
    derivatives(sys, t);

    if (itime == 1) {
      for (int i = 0; i < sys->NumberOfFluidParticles; i++) {
        sys->localDensity[i] = sys->density[i] + 0.5 * dt * sys->ddensitydt[i] + sys->densityFluctuation[i];
        sys->density[i] += 0.5 * dt * sys->ddensitydt[i];
        sys->localPressure[i] = sys->DynamicPressure[i] + 0.5 * dt * sys->dpdt[i] + sys->pressureFluctuation[i];
        sys->DynamicPressure[i] += 0.5 * dt * sys->dpdt[i];
      }
      for (int i = 0; i < sys->NumberOfFluidParticles; i++) {
        for (int d = 0; d < sys->dim; d++) {
          sys->Velocity_xsph[i][d] = sys->Velocity[i][d] + 0.5 * dt * sys->dvdt[i][d] + sys->epsilon * sys->velocityFluctuation[i][d];
          sys->localVelocity[i][d] = sys->Velocity[i][d] + 0.5 * dt * sys->dvdt[i][d] + sys->epsilon * sys->velocityFluctuation[i][d];
          sys->Velocity[i][d] += 0.5 * dt * sys->dvdt[i][d];
          sys->Position[i][d] += dt * sys->Velocity[i][d];
        }
      }
    } else {
      for (int i = 0; i < sys->NumberOfFluidParticles; i++) {
        sys->localDensity[i] = sys->density_min[i] + dt * sys->ddensitydt[i] + sys->densityFluctuation[i];
        sys->density[i] = sys->density_min[i] + dt * sys->ddensitydt[i];
        sys->localPressure[i] = sys->DynamicPressure_min[i] + dt * sys->dpdt[i] + sys->pressureFluctuation[i];
        sys->DynamicPressure[i] = sys->DynamicPressure_min[i] + dt * sys->dpdt[i];
      }
      for (int i = 0; i < sys->NumberOfFluidParticles; i++) {
        for (int d = 0; d < sys->dim; d++) {
          sys->Velocity_xsph[i][d] = sys->Velocity_min[i][d] + dt * sys->dvdt[i][d] + sys->epsilon * sys->velocityFluctuation[i][d];
          sys->localVelocity[i][d] = sys->Velocity_min[i][d] + dt * sys->dvdt[i][d] + sys->epsilon * sys->velocityFluctuation[i][d];
          sys->Velocity[i][d] = sys->Velocity_min[i][d] + dt * sys->dvdt[i][d];
          sys->Position[i][d] += dt * sys->Velocity[i][d];
        }
      }
    }
  }
  if (chdir(cwd)) return -1;
  return 0;
}

/* counts: Nf, Ns, Nfixed, Nmoving, Nb, niac, MaxN, itime */
void ref_counts(const ref_run *run, int out[9])
{
  const System *s = run->sys;
  out[8] = s->NumberOfVirtualParticles;
  out[0] = s->NumberOfFluidParticles;
  out[1] = s->NumberOfSolidParticles;
  out[2] = s->NumberOfFixedBoundaryParticles;
  out[3] = s->NumberOfMovingBoundaryParticles;
  out[4] = s->NumberOfBoundaryParticles;
  out[5] = s->NumberOfInteractingParticles;
  out[6] = s->MaxNumberOfParticles;
  out[7] = run->itime;
}

/* derived scalars: dt, c0, B, eta, hsml[0], rho0, gamma, g, k_spring, c_damp,
   kappa0, mu0, epsilon, dx, omega, stroke */
void ref_scalars(const ref_run *run, double out[16])
{
  const System *s = run->sys;
  out[0] = s->timeStep;
  out[1] = s->SpeedOfSound;
  out[2] = s->CompressionFactor;
  out[3] = s->eta;
  out[4] = s->hsml[0];
  out[5] = s->density0;
  out[6] = s->AdiabaticConstant;
  out[7] = s->Gravity;
  out[8] = s->springConstant0;
  out[9] = s->dampingConstant0;
  out[10] = s->thermalDiffusivity0;
  out[11] = s->viscosity0;
  out[12] = s->epsilon;
  out[13] = s->dx;
  out[14] = s->omega;
  out[15] = s->stroke;
}

static double **vec_field(System *s, const char *name)
{
  if (!strcmp(name, "Position")) return s->Position;
  if (!strcmp(name, "Velocity")) return s->Velocity;
  if (!strcmp(name, "localVelocity")) return s->localVelocity;
  if (!strcmp(name, "Velocity_min")) return s->Velocity_min;
  if (!strcmp(name, "dvdt")) return s->dvdt;
  if (!strcmp(name, "dvdt_approx")) return s->dvdt_approx;
  if (!strcmp(name, "velocityFluctuation")) return s->velocityFluctuation;
  if (!strcmp(name, "dwcdx")) return s->dwcdx;
  return NULL;
}

static double *scal_field(System *s, const char *name)
{
  if (!strcmp(name, "density")) return s->density;
  if (!strcmp(name, "DynamicPressure")) return s->DynamicPressure;
  if (!strcmp(name, "localDensity")) return s->localDensity;
  if (!strcmp(name, "localPressure")) return s->localPressure;
  if (!strcmp(name, "density_min")) return s->density_min;
  if (!strcmp(name, "DynamicPressure_min")) return s->DynamicPressure_min;
  if (!strcmp(name, "ddensitydt")) return s->ddensitydt;
  if (!strcmp(name, "dpdt")) return s->dpdt;
  if (!strcmp(name, "ddensitydt_approx")) return s->ddensitydt_approx;
  if (!strcmp(name, "dpdt_approx")) return s->dpdt_approx;
  if (!strcmp(name, "densityFluctuation")) return s->densityFluctuation;
  if (!strcmp(name, "pressureFluctuation")) return s->pressureFluctuation;
  if (!strcmp(name, "Pressure")) return s->Pressure;
  if (!strcmp(name, "mass")) return s->mass;
  if (!strcmp(name, "hsml")) return s->hsml;
  if (!strcmp(name, "rij2")) return s->rij2;
  if (!strcmp(name, "w")) return s->w;
  if (!strcmp(name, "spongeFactor")) return s->spongeFactor;
  return NULL;
}

/* Copies n entries of a named field starting at `first`; vectors come out as
   [n][2] (the reference's own layout).  Returns the number of doubles copied,
   or -1 for an unknown name. */
long ref_get(ref_run *run, const char *name, int first, int n, double *out)
{
  double **v = vec_field(run->sys, name);
  if (v) {
    memcpy(out, v[0] + 2L * first, sizeof(double) * 2L * n);
    return 2L * n;
  }
  double *a = scal_field(run->sys, name);
  if (a) {
    memcpy(out, a + first, sizeof(double) * (size_t)n);
    return n;
  }
  return -1;
}

long ref_set(ref_run *run, const char *name, int first, int n, const double *in)
{
  double **v = vec_field(run->sys, name);
  if (v) {
    memcpy(v[0] + 2L * first, in, sizeof(double) * 2L * n);
    return 2L * n;
  }
  double *a = scal_field(run->sys, name);
  if (a) {
    memcpy(a + first, in, sizeof(double) * (size_t)n);
    return n;
  }
  return -1;
}

int ref_get_itype(ref_run *run, int first, int n, int *out)
{
  memcpy(out, run->sys->itype + first, sizeof(int) * (size_t)n);
  return n;
}

/* The interaction pairs of the last derivatives() call. */
int ref_pairs(ref_run *run, int *i_pair, int *j_pair)
{
  const int niac = run->sys->NumberOfInteractingParticles;
  memcpy(i_pair, run->sys->i_pair, sizeof(int) * (size_t)niac);
  memcpy(j_pair, run->sys->j_pair, sizeof(int) * (size_t)niac);
  return niac;
}

System *ref_system(ref_run *run) { return run->sys; }
