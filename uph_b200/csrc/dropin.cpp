// libuph_sph: derivatives() and SearchNeighbors() with the reference's own
// signatures, on top of the C ABI in uph.h.  The caller keeps the rest of
// its libSPH (inputbp.c, inoutflow.c, ...) and its driver; see uph_system.h.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "uph.h"
#include "uph_system.h"

extern "C" {
// the caller's own libSPH provides these (inputbp.c:12, inoutflow.c:14);
// weak, so a caller without a libSPH can load the library and register its
// own through uph_dropin_set_callbacks instead
void inputbp(System *sys, double t) __attribute__((weak));
void inoutflow(System *sys) __attribute__((weak));
}

namespace {

struct DropIn {
  uph_sim *sim = nullptr;
  uph_params p;
  // the System whose arrays past its particles were zeroed
  const System *zeroed = nullptr;
  int zeroed_n = 0, zeroed_max = 0;
  int pair_export = 2;  // uph_dropin_set_pair_export
  // uph_dropin_set_callbacks; null: the libSPH functions linked with the caller
  void (*inputbp)(System *, double) = nullptr;
  void (*inoutflow)(System *) = nullptr;
};

DropIn g;

[[noreturn]] void die(const char *where, uph_status s)
{
  // the reference reports errors with printf + exit(1) (System.c:55-59)
  printf("%s: %s: %s\n", where, uph_status_string(s), uph_last_error());
  fflush(stdout);
  exit(1);
}

// System -> uph_params (the fields CreateSystem filled, System.c:60-335)
void params_from_system(const System *sys, uph_params *p)
{
  memset(p, 0, sizeof *p);
  p->profile = UPH_PROFILE_REF;
  p->precision = UPH_PREC_FP64;
  p->n_fluid = sys->NumberOfFluidParticles;
  p->n_solid = sys->NumberOfSolidParticles;
  p->n_fixed = sys->NumberOfFixedBoundaryParticles;
  p->n_moving = sys->NumberOfMovingBoundaryParticles;
  p->stroke = sys->stroke;
  p->wave_period = sys->wavePeriod;
  p->local_depth = sys->LocalDepth;
  p->flat_bottom_length = sys->FlatBottomLength;
  p->density0 = sys->density0;
  p->adiabatic_constant = sys->AdiabaticConstant;
  p->gravity = sys->Gravity;
  p->dx = sys->dx;
  p->dy = sys->dy;
  p->dim = sys->dim;
  p->viscosity0 = sys->viscosity0;
  p->mach_number = sys->machNumber;
  p->peclet_number = sys->pecletNumber;
  p->epsilon = sys->epsilon;
  p->alpha = sys->alpha;
  p->virtual_type = sys->virtualType;
  p->print_step = sys->printStep;
  p->screen_step = sys->screenStep;
  p->time_step = sys->timeStep;
  p->lid_velocity = sys->lidVelocity;
  p->near_neighbor = sys->nearNeighbor;
  p->select_boundary_force = sys->selectBoundaryForce;
  p->lennard_select = sys->lennardSelect;
  p->spring_constant0 = sys->springConstant0;
  p->damping_constant0 = sys->dampingConstant0;
  p->flag_init_simul = sys->flagInitSimul;
  p->gravity_flag = sys->gravityFlag;
  p->thermal_diffusivity0 = sys->thermalDiffusivity0;
  p->moving_boundary = sys->movingBoundary;
  p->number_of_initialization_steps = sys->NumberOfInitializationSteps;
  p->pressure_probe_x = sys->pressureProbeX;
  p->pressure_probe_y = sys->pressureProbeY;
  p->stress_type = sys->stressType;
  p->dissipation_control_volume = sys->disspationControlVolume;
  p->speed_of_sound = sys->SpeedOfSound;
  p->compression_factor = sys->CompressionFactor;
  p->omega = sys->omega;
  p->eta = sys->eta;
  p->h = sys->hsml[0];
  p->lennard_coefficient = sys->LennardCoefficient;
  p->sponge_factor0 = sys->spongeFactor0;
  p->sponge_position0 = sys->spongePosition0;
  p->wave_absorption = sys->waveAbsorption;
  p->av_alpha = sys->alpha;
  p->knn_cap = 40;  // SearchNeighbors' k (derivatives.c:1085)
}

// The library uses one smoothing length, one viscosity and one diffusivity;
// input.c:105-119 and inputbp.c:285-299 give every particle the same values.
void check_uniform(const System *sys, int n)
{
  const double h = sys->hsml[0], mu = sys->viscosity[0], k = sys->thermalDiffusivity[0];
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (int i = 0; i < n; i++)
    bad |= sys->hsml[i] != h || sys->viscosity[i] != mu || sys->thermalDiffusivity[i] != k;
  if (bad)
    for (int i = 0; i < n; i++)
      if (sys->hsml[i] != h || sys->viscosity[i] != mu || sys->thermalDiffusivity[i] != k) {
        printf("derivatives: particle %d has its own hsml/viscosity/thermalDiffusivity; "
               "the GPU path needs the uniform values input() assigns\n", i);
        exit(1);
      }
  if (mu != sys->viscosity0 || k != sys->thermalDiffusivity0) {
    printf("derivatives: per-particle viscosity/thermalDiffusivity differ from viscosity0/thermalDiffusivity0\n");
    exit(1);
  }
}

// The simulation for this System's parameters.  Its cell-grid domain is the
// particles' bounding box with room to move; the box is only measured when
// the simulation is made, or with `remeasure` after an upload found a
// particle outside the domain.
void ensure_sim(const System *sys, int n, bool remeasure)
{
  uph_params p;
  params_from_system(sys, &p);
  bool same = g.sim != nullptr;
  if (same) {
    const uph_params &q = g.p;
    same = q.n_fluid == p.n_fluid && q.n_solid == p.n_solid && q.n_fixed == p.n_fixed && q.n_moving == p.n_moving &&
           q.h == p.h && q.time_step == p.time_step &&
           memcmp(&q.stroke, &p.stroke, offsetof(uph_params, domain_lo) - offsetof(uph_params, stroke)) == 0;
  }
  if (same && !remeasure) return;
  double x0 = sys->Position[0][0], x1 = x0, y0 = sys->Position[0][1], y1 = y0;
#pragma omp parallel for schedule(static) reduction(min : x0, y0) reduction(max : x1, y1)
  for (int i = 1; i < n; i++) {
    x0 = fmin(x0, sys->Position[i][0]);
    x1 = fmax(x1, sys->Position[i][0]);
    y0 = fmin(y0, sys->Position[i][1]);
    y1 = fmax(y1, sys->Position[i][1]);
  }
  const double lo[2] = {x0, y0}, hi[2] = {x1, y1};
  if (same && lo[0] >= g.p.domain_lo[0] && lo[1] >= g.p.domain_lo[1] && hi[0] <= g.p.domain_hi[0] &&
      hi[1] <= g.p.domain_hi[1])
    return;
  if (g.sim) uph_sim_destroy(g.sim);
  g.sim = nullptr;
  for (int d = 0; d < 2; d++) {
    const double ext = hi[d] - lo[d];
    p.domain_lo[d] = lo[d] - 0.5 * ext - 8.0 * p.h;
    p.domain_hi[d] = hi[d] + 0.5 * ext + 8.0 * p.h;
  }
  uph_status s = uph_sim_create(&p, &g.sim);
  if (s != UPH_OK) die("derivatives", s);
  g.p = p;
}

// The virtual mirror particles (derivatives.c:3194-4192) as the reference
// leaves them in the System: rows from Nf + Ns + Nb on, each a copy of its
// fluid particle taken before this call's equation of state, with the
// mirrored position (computed on the device) and velocities, itype 4.
void write_virtual_rows(System *sys, int n)
{
  int64_t nv = 0;
  uph_status s = uph_sim_virtual(g.sim, 0, nullptr, nullptr, nullptr, &nv);
  if (s != UPH_OK) die("derivatives", s);
  sys->NumberOfVirtualParticles = (int)nv;
  if (nv == 0) return;
  if (n + nv > sys->MaxNumberOfParticles) {
    printf("derivatives: %lld virtual particles do not fit in MaxNumberOfParticles = %d\n", (long long)nv,
           sys->MaxNumberOfParticles);
    fflush(stdout);
    exit(1);
  }
  std::vector<double> pos(2 * (size_t)nv);
  std::vector<int32_t> src((size_t)nv), kind((size_t)nv);
  s = uph_sim_virtual(g.sim, nv, pos.data(), src.data(), kind.data(), &nv);
  if (s != UPH_OK) die("derivatives", s);
  const double sl = sys->slope, denoms = 1 + sl * sl, nums = 1 - sl * sl;
  for (int64_t k = 0; k < nv; k++) {
    const int ii = n + (int)k, i = src[k];
    sys->Position[ii][0] = pos[2 * k];
    sys->Position[ii][1] = pos[2 * k + 1];
    for (double **v : {sys->Velocity, sys->Velocity_xsph, sys->localVelocity}) {
      const double vx = v[i][0], vy = v[i][1];
      switch (kind[k]) {
        case 0:  // left and right walls
        case 1:
          v[ii][0] = -vx;
          v[ii][1] = vy;
          break;
        case 2:  // bottom and top
        case 3:
          v[ii][0] = vx;
          v[ii][1] = -vy;
          break;
        case 4:  // corners
        case 5:
          v[ii][0] = -vx;
          v[ii][1] = -vy;
          break;
        default:  // the slope
          v[ii][0] = (nums * vx + 2.0 * sl * vy) / denoms;
          v[ii][1] = (2.0 * sl * vx - nums * vy) / denoms;
          break;
      }
    }
    for (double *f : {sys->mass, sys->density, sys->Pressure, sys->Energy, sys->hsml, sys->normalizationFactor,
                      sys->DynamicPressure, sys->localDensity, sys->localPressure, sys->vorticity,
                      sys->thermalDiffusivity})
      f[ii] = f[i];
    sys->itype[ii] = 4;
  }
}

}  // namespace

extern "C" void derivatives(System *sys, double t)
{
  const int nf = sys->NumberOfFluidParticles;
  const int nall = nf + sys->NumberOfSolidParticles + sys->NumberOfBoundaryParticles;
  // derivatives.c:3147-3157 zeroes the rate arrays (MaxNumberOfParticles
  // long; the stress arrays feed stressType 2 only).  The fluid entries are
  // overwritten below; the other particles' are zeroed every call; entries
  // past the particles, which nothing writes, once per System.
  const size_t M = (size_t)sys->MaxNumberOfParticles;
  const bool first = g.zeroed != sys || g.zeroed_n != nall || g.zeroed_max != sys->MaxNumberOfParticles;
  const size_t z0 = (size_t)nf, z1 = first ? M : (size_t)nall;
  if (z1 > z0) {
    for (double *v : {sys->ddensitydt, sys->dpdt, sys->ddensitydt_approx, sys->dpdt_approx})
      memset(v + z0, 0, sizeof(double) * (z1 - z0));
    for (double *v : {sys->dvdt[0], sys->dvdt_approx[0]}) memset(v + 2 * z0, 0, sizeof(double) * 2 * (z1 - z0));
  }
  g.zeroed = sys;
  g.zeroed_n = nall;
  g.zeroed_max = sys->MaxNumberOfParticles;
  void (*cb_inoutflow)(System *) = g.inoutflow ? g.inoutflow : inoutflow;
  void (*cb_inputbp)(System *, double) = g.inputbp ? g.inputbp : inputbp;
  if (!cb_inoutflow || !cb_inputbp) {
    printf("derivatives: no inputbp()/inoutflow(): link the caller's libSPH or call uph_dropin_set_callbacks\n");
    fflush(stdout);
    exit(1);
  }
  if (t > 0) cb_inoutflow(sys);  // derivatives.c:3162-3164
  cb_inputbp(sys, t);            // derivatives.c:3168: re-reads the boundary decks, moves walls
  // derivatives.c:3171-3182 only feeds inoutflow's inflow branch, whose
  // threshold (x > 5000.1, inoutflow.c:26) no deck reaches; it is not repeated.
  sys->inflowParticles = 0;
  const int nb = sys->NumberOfBoundaryParticles, ns = sys->NumberOfSolidParticles;
  for (int i = 0; i < nb; i++)  // derivatives.c:3187-3191
    for (int d = 0; d < 2; d++) sys->Velocity_xsph[nf + ns + i][d] = sys->Velocity[nf + ns + i][d];
  sys->NumberOfVirtualParticles = 0;
  const int n = nf + ns + nb;
  check_uniform(sys, n);
  if (sys->flagInitSimul == 0 && sys->NumberOfFrozenParticles > 0) {
    printf("derivatives: frozen particles (FrozenParticle.dat) are not supported\n");
    fflush(stdout);
    exit(1);
  }
  ensure_sim(sys, n, false);

  uph_state in;
  memset(&in, 0, sizeof in);
  in.Position = sys->Position[0];
  in.Velocity = sys->Velocity[0];
  in.localVelocity = sys->localVelocity[0];
  in.density = sys->density;
  in.localDensity = sys->localDensity;
  in.DynamicPressure = sys->DynamicPressure;
  in.localPressure = sys->localPressure;
  in.mass = sys->mass;
  in.itype = sys->itype;
  in.spongeFactor = sys->spongeFactor;
  uph_status s = uph_sim_upload(g.sim, &in, 0);
  if (s == UPH_OUT_OF_DOMAIN) {
    // a particle left the cell grid made for an earlier call: measure again
    ensure_sim(sys, n, true);
    s = uph_sim_upload(g.sim, &in, 0);
  }
  if (s != UPH_OK) die("derivatives", s);
  s = uph_sim_derivatives(g.sim, t);
  if (s != UPH_OK) die("derivatives", s);
  write_virtual_rows(sys, n);
  uph_state out;
  memset(&out, 0, sizeof out);
  out.ddensitydt = sys->ddensitydt;
  out.dpdt = sys->dpdt;
  out.dvdt = sys->dvdt[0];
  out.ddensitydt_approx = sys->ddensitydt_approx;
  out.dpdt_approx = sys->dpdt_approx;
  out.dvdt_approx = sys->dvdt_approx[0];
  out.densityFluctuation = sys->densityFluctuation;
  out.pressureFluctuation = sys->pressureFluctuation;
  out.velocityFluctuation = sys->velocityFluctuation[0];
  out.Pressure = sys->Pressure;
  if (sys->flagInitSimul == 0) {
    // particle packing resets the fluid's density and pressure
    // (InitialDensityAndPressure, derivatives.c:3056-3066) and computes no
    // equation of state
    out.density = sys->density;
    out.DynamicPressure = sys->DynamicPressure;
    out.Pressure = nullptr;
  }
  s = uph_sim_download(g.sim, &out);
  if (s != UPH_OK) die("derivatives", s);
  // LocalDensity/Pressure/VelocityFluctuation zero the boundary entries (derivatives.c:2062-2066, 2103-2106, 2140-2143)
  for (int i = nf; i < nf + nb; i++) {
    sys->densityFluctuation[i] = 0.0;
    sys->pressureFluctuation[i] = 0.0;
    sys->velocityFluctuation[i][0] = 0.0;
    sys->velocityFluctuation[i][1] = 0.0;
  }
  // the pair count, and TotalKineticEnergy (derivatives.c:2254-2264): the
  // reference's terms over the fluid, reduced on the device from the state
  // this call uploaded (a fixed grid of partial sums, so the result does not
  // depend on anything but the state; it can differ from the serial sum in
  // the last bits)
  uph_stats st;
  s = uph_sim_stats(g.sim, &st);
  if (s != UPH_OK) die("derivatives", s);
  sys->totalKineticEnergy = st.kinetic_energy;
  sys->potentialEnergy = st.potential_energy;
  // pair list (CalculateKernel's outputs, derivatives.c:1076-1105)
  int64_t niac = 0;
  if (g.pair_export == 0) {
    niac = st.niac;
  } else {
    const bool all = g.pair_export >= 2;
    s = uph_sim_pairs(g.sim, sys->MaxNumberOfParticles, sys->i_pair, sys->j_pair, sys->rij2, all ? sys->w : nullptr,
                      all ? sys->dwcdx[0] : nullptr, &niac);
    if (s != UPH_OK) die("derivatives", s);
  }
  sys->NumberOfInteractingParticles = (int)niac;
  // ApproximateVortcity (derivatives.c:2840-2885), printed by output()
  if (sys->flagInitSimul == 1 && sys->approxVorticity) {
    s = uph_sim_approx_vorticity(g.sim, sys->approxVorticity);
    if (s != UPH_OK) die("derivatives", s);
    for (int i = nf; i < nf + nb; i++) sys->approxVorticity[i] = 0.0;  // derivatives.c:2843-2846
  }
}

extern "C" int SearchNeighbors(const double **Position, int *i_pair, int *j_pair, double *rij2,
                               const int NumberOfFluidParticles, const int NumberOfParticles, int ParticleBoundary,
                               const int NumberOfNeighbors, const double dist)
{
  int64_t niac = 0;
  // the caller sizes the pair arrays by MaxNumberOfParticles; it is not passed, so
  // ask for the count first and then fill
  uph_status s = uph_search_neighbors(Position[0], NumberOfFluidParticles, NumberOfParticles, ParticleBoundary,
                                      NumberOfNeighbors, dist, 0, nullptr, nullptr, nullptr, &niac);
  if (s != UPH_OK && s != UPH_NEIGHBOR_OVERFLOW) die("SearchNeighbors", s);
  s = uph_search_neighbors(Position[0], NumberOfFluidParticles, NumberOfParticles, ParticleBoundary,
                           NumberOfNeighbors, dist, niac, i_pair, j_pair, rij2, &niac);
  if (s != UPH_OK) die("SearchNeighbors", s);
  return (int)niac;
}

extern "C" void uph_dropin_set_pair_export(int level)
{
  g.pair_export = level < 0 ? 0 : level > 2 ? 2 : level;
}

extern "C" void uph_dropin_set_callbacks(void (*inputbp_fn)(System *, double), void (*inoutflow_fn)(System *))
{
  g.inputbp = inputbp_fn;
  g.inoutflow = inoutflow_fn;
}
