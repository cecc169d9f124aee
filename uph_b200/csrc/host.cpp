// Host-side parts of the C ABI: parameters.dat parsing and the derived
// quantities of CreateSystem, deck reading, status strings and the
// thread-local error message.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "uph_internal.cuh"

namespace uph {

std::string &last_error()
{
  static thread_local std::string msg;
  return msg;
}

uph_status fail(uph_status s, const std::string &msg)
{
  last_error() = msg;
  return s;
}

uph_status cuda_fail(cudaError_t e, const char *what)
{
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return fail(UPH_OUT_OF_MEMORY, m);
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return fail(UPH_NO_DEVICE, m);
  return fail(UPH_CUDA_ERROR, m);
}

}  // namespace uph

using namespace uph;

extern "C" const char *uph_status_string(uph_status s)
{
  switch (s) {
  case UPH_OK: return "UPH_OK";
  case UPH_BAD_ARG: return "UPH_BAD_ARG";
  case UPH_OUT_OF_DOMAIN: return "UPH_OUT_OF_DOMAIN";
  case UPH_NEIGHBOR_OVERFLOW: return "UPH_NEIGHBOR_OVERFLOW";
  case UPH_NAN: return "UPH_NAN";
  case UPH_TIMEOUT: return "UPH_TIMEOUT";
  case UPH_CUDA_ERROR: return "UPH_CUDA_ERROR";
  case UPH_NO_DEVICE: return "UPH_NO_DEVICE";
  case UPH_UNSUPPORTED: return "UPH_UNSUPPORTED";
  case UPH_OUT_OF_MEMORY: return "UPH_OUT_OF_MEMORY";
  case UPH_IO_ERROR: return "UPH_IO_ERROR";
  }
  return "UPH_UNKNOWN";
}

extern "C" const char *uph_last_error(void) { return last_error().c_str(); }

// System.c:292-335 and input.c:107
extern "C" uph_status uph_params_derive(uph_params *p, double eta_override)
{
  if (!p) return fail(UPH_BAD_ARG, "uph_params_derive: NULL params");
  if (!(p->mach_number > 0) || !(p->adiabatic_constant > 0) || p->near_neighbor < 0)
    return fail(UPH_BAD_ARG, "uph_params_derive: machNumber and AdiabaticConstant must be positive");
  if (p->moving_boundary == 2)
    p->speed_of_sound = sqrt(2.0 * p->gravity * p->local_depth) / p->mach_number;
  else
    p->speed_of_sound = sqrt(p->gravity * p->local_depth) / p->mach_number;
  p->compression_factor = (1. / p->adiabatic_constant) * p->density0 * p->speed_of_sound * p->speed_of_sound;
  p->omega = p->wave_period != 0.0 ? 2.0 * M_PI / p->wave_period : 0.0;
  p->eta = sqrt(p->near_neighbor / (4.0 * M_PI));
  if (eta_override > 0.0) p->eta = eta_override;
  p->h = p->eta * p->dx;
  p->lennard_coefficient = p->gravity * p->local_depth;
  p->sponge_factor0 = 0.2;
  p->sponge_position0 = 7.0;
  p->wave_absorption = 1;
  return UPH_OK;
}

extern "C" uph_status uph_params_from_file(const char *path, double eta_override, uph_params *out)
{
  if (!path || !out) return fail(UPH_BAD_ARG, "uph_params_from_file: NULL argument");
  FILE *f = fopen(path, "r");
  if (!f) return fail(UPH_IO_ERROR, std::string("cannot find parameter file ") + path);
  uph_params p;
  memset(&p, 0, sizeof p);
  // the 34 fields of System.c:60-94, in file order
  int got = fscanf(f, "%lf %lf %lf %lf %lf %lf %lf %lf %lf %d %lf %lf %lf %lf %lf %d %d %d %lf %lf %d %d %lf %lf %lf "
                      "%d %d %lf %d %d %lf %lf %d %d",
                   &p.stroke, &p.wave_period, &p.local_depth, &p.flat_bottom_length, &p.density0,
                   &p.adiabatic_constant, &p.gravity, &p.dx, &p.dy, &p.dim, &p.viscosity0, &p.mach_number,
                   &p.peclet_number, &p.epsilon, &p.alpha, &p.virtual_type, &p.print_step, &p.screen_step,
                   &p.time_step, &p.lid_velocity, &p.near_neighbor, &p.select_boundary_force, &p.lennard_select,
                   &p.spring_constant0, &p.damping_constant0, &p.flag_init_simul, &p.gravity_flag,
                   &p.thermal_diffusivity0, &p.moving_boundary, &p.number_of_initialization_steps,
                   &p.pressure_probe_x, &p.pressure_probe_y, &p.stress_type, &p.dissipation_control_volume);
  fclose(f);
  if (got != 34) return fail(UPH_IO_ERROR, std::string(path) + ": expected 34 values, read " + std::to_string(got));
  p.av_alpha = p.alpha;
  uph_status s = uph_params_derive(&p, eta_override);
  if (s != UPH_OK) return s;
  *out = p;
  return UPH_OK;
}

namespace {

// One particle file: a count line then 12 columns per row (input.c:59-71).
uph_status read_block(const std::string &path, bool required, std::vector<double> &rows, int &count)
{
  rows.clear();
  count = 0;
  FILE *f = fopen(path.c_str(), "r");
  if (!f) {
    if (required) return fail(UPH_IO_ERROR, "cannot find " + path);
    return UPH_OK;
  }
  if (fscanf(f, "%d", &count) != 1 || count < 0) {
    fclose(f);
    if (!required) { count = 0; return UPH_OK; }
    return fail(UPH_IO_ERROR, path + ": missing particle count");
  }
  rows.resize((size_t)count * 12);
  for (int i = 0; i < count; i++) {
    double *r = &rows[(size_t)i * 12];
    int it = 0;
    int got = fscanf(f, "%lf %lf %lf %lf %lf %lf %lf %lf %lf %d %lf %lf", &r[0], &r[1], &r[2], &r[3], &r[4], &r[5],
                     &r[6], &r[7], &r[8], &it, &r[10], &r[11]);
    if (got != 12) {
      fclose(f);
      return fail(UPH_IO_ERROR, path + ": row " + std::to_string(i) + " has " + std::to_string(got) + " of 12 values");
    }
    r[9] = it;
  }
  fclose(f);
  return UPH_OK;
}

}  // namespace

// input.c:22-164 and inputbp.c:12-191, 285-290: the state a fresh deck has at
// the first derivatives() call.
extern "C" uph_status uph_deck_read(const char *deck_dir, double eta_override, uph_params *p, uph_state *st)
{
  if (!deck_dir || !p) return fail(UPH_BAD_ARG, "uph_deck_read: NULL argument");
  const std::string dir(deck_dir);
  uph_params q;
  uph_status s = uph_params_from_file((dir + "/parameters.dat").c_str(), eta_override, &q);
  if (s != UPH_OK) return s;
  std::vector<double> blk[4];
  int cnt[4];
  const char *names[4] = {"FluidParticle.dat", "SolidParticle.dat", "FixedBoundaryParticle.dat",
                          "MovingBoundaryParticle.dat"};
  for (int k = 0; k < 4; k++) {
    s = read_block(dir + "/" + names[k], k != 1, blk[k], cnt[k]);
    if (s != UPH_OK) return s;
  }
  q.n_fluid = cnt[0];
  q.n_solid = cnt[1];
  q.n_fixed = cnt[2];
  q.n_moving = cnt[3];
  q.profile = p->profile;
  q.precision = p->precision;
  q.knn_cap = p->knn_cap;
  if (p->av_alpha != 0.0) q.av_alpha = p->av_alpha;
  memcpy(q.domain_lo, p->domain_lo, sizeof q.domain_lo);
  memcpy(q.domain_hi, p->domain_hi, sizeof q.domain_hi);
  *p = q;
  if (!st) return UPH_OK;
  const int nf = cnt[0];
  int idx = 0;
  for (int k = 0; k < 4; k++)
    for (int i = 0; i < cnt[k]; i++, idx++) {
      const double *r = &blk[k][(size_t)i * 12];
      if (st->Position) { st->Position[2 * idx] = r[0]; st->Position[2 * idx + 1] = r[1]; }
      if (st->Velocity) { st->Velocity[2 * idx] = r[2]; st->Velocity[2 * idx + 1] = r[3]; }
      if (st->density) st->density[idx] = r[4];
      if (st->DynamicPressure) st->DynamicPressure[idx] = r[5];
      if (st->mass) st->mass[idx] = r[6];
      if (st->itype) st->itype[idx] = (int32_t)r[9];
      if (st->localVelocity) { st->localVelocity[2 * idx] = r[10]; st->localVelocity[2 * idx + 1] = r[11]; }
      if (st->localDensity) st->localDensity[idx] = q.density0;  // input.c:109, inputbp.c:289
      if (st->localPressure) st->localPressure[idx] = 0.0;       // input.c:110, inputbp.c:290
      if (idx < nf) {
        if (st->density_min) st->density_min[idx] = r[4];          // sph.cc:81
        if (st->DynamicPressure_min) st->DynamicPressure_min[idx] = r[5];  // sph.cc:83
        if (st->Velocity_min) { st->Velocity_min[2 * idx] = 0.0; st->Velocity_min[2 * idx + 1] = 0.0; }
        if (st->spongeFactor)  // input.c:137-144
          st->spongeFactor[idx] = r[0] >= q.sponge_position0 ? q.sponge_factor0 : 0.0;
      }
    }
  double *zero_fluid[] = {st->ddensitydt, st->dpdt, st->ddensitydt_approx, st->dpdt_approx, st->densityFluctuation,
                          st->pressureFluctuation};
  for (double *z : zero_fluid)
    if (z) memset(z, 0, sizeof(double) * (size_t)nf);
  double *zero_vec[] = {st->dvdt, st->dvdt_approx, st->velocityFluctuation};
  for (double *z : zero_vec)
    if (z) memset(z, 0, sizeof(double) * 2 * (size_t)nf);
  if (st->Pressure) memset(st->Pressure, 0, sizeof(double) * (size_t)idx);
  return UPH_OK;
}

namespace {

// opens `name` in `dir` with the reference's mode and a large buffer
FILE *open_in(const std::string &dir, const char *name, const char *mode, std::vector<char> *buf = nullptr)
{
  FILE *f = fopen((dir + "/" + name).c_str(), mode);
  if (f && buf) setvbuf(f, buf->data(), _IOFBF, buf->size());
  return f;
}

}  // namespace

// output() of output.c:19-140 for the files the hot path has values for; the
// formats are the reference's, character for character
extern "C" uph_status uph_write_output(const char *directory, int32_t itime, const uph_params *p, const uph_state *st,
                                       const int32_t *dam_gate_flag, const uph_diagnostics *diag)
{
  if (!directory || !p || !st || !diag) return fail(UPH_BAD_ARG, "uph_write_output: NULL argument");
  if (!st->Position || !st->Velocity || !st->density || !st->mass || !st->DynamicPressure || !st->itype ||
      !st->localDensity || !st->localVelocity)
    return fail(UPH_BAD_ARG, "uph_write_output: the state needs Position, Velocity, localVelocity, density, "
                             "localDensity, DynamicPressure, mass and itype");
  const std::string dir(directory);
  const int nf = p->n_fluid;
  const int n = p->n_fluid + p->n_solid + p->n_fixed + p->n_moving;
  const double t = p->time_step * itime;
  std::vector<char> buf(1 << 22);
  char name[64];
  snprintf(name, sizeof name, "out%d.dat", itime);
  FILE *f = open_in(dir, name, "w+", &buf);
  if (!f) return fail(UPH_IO_ERROR, "uph_write_output: cannot open " + dir + "/" + name);
  for (int i = 0; i < n; i++) {
    fprintf(f, "%d ", i);
    fprintf(f, "\t%.10lf\t%.10lf", st->Position[2 * i], st->Position[2 * i + 1]);
    fprintf(f, "\t%.10lf\t%.10lf", st->Velocity[2 * i], st->Velocity[2 * i + 1]);
    fprintf(f, "\t%.10lf\t%.10lf\t%.10lf\t%.10lf\t%d\t%.10lf\t%d\t%.10lf\t%.10lf\n", st->density[i], st->mass[i], p->h,
            st->DynamicPressure[i], dam_gate_flag ? dam_gate_flag[i] : 0, 0.0, st->itype[i], 0.0,
            st->localDensity[i]);
  }
  bool ok = fclose(f) == 0;
  if ((f = open_in(dir, "TotalKineticEnergy.dat", "a"))) {
    fprintf(f, "%.10lf\t%.10lf %.10lf\n", t, diag->kinetic_energy, diag->potential_energy);
    ok = fclose(f) == 0 && ok;
  } else {
    ok = false;
  }
  if ((f = open_in(dir, "PointPressure.dat", "a"))) {
    fprintf(f, "%.10lf\t%.10lf\t%d\t%.10lf\t%.10lf\n", t, diag->point_pressure, diag->point_neighbors,
            diag->pressure_norm, diag->point_pressure_two);
    ok = fclose(f) == 0 && ok;
  } else {
    ok = false;
  }
  if ((f = open_in(dir, "PointPressureTwo.dat", "a"))) {
    fprintf(f, "%.10lf\t%d\t%.10lf\n", t, diag->point_neighbors_two, diag->point_pressure_two);
    ok = fclose(f) == 0 && ok;
  } else {
    ok = false;
  }
  if (itime == p->number_of_initialization_steps) {
    if ((f = open_in(dir, "FluidParticleInit.dat", "a", &buf))) {
      fprintf(f, "%d\n", nf);
      for (int i = 0; i < nf; i++) {
        fprintf(f, "%.10lf\t%.10lf\t", st->Position[2 * i], st->Position[2 * i + 1]);
        fprintf(f, "%.10lf\t%.10lf\t", st->Velocity[2 * i], st->Velocity[2 * i + 1]);
        fprintf(f, "%.10lf\t%.10lf\t%.10lf\t%.10lf\t%.10lf\t%d\t%.10lf\t%.10lf\n", st->density[i],
                st->DynamicPressure[i], st->mass[i], 0.0, 0.0, st->itype[i], st->localVelocity[2 * i],
                st->localVelocity[2 * i + 1]);
      }
      ok = fclose(f) == 0 && ok;
    } else {
      ok = false;
    }
  }
  if (!ok) return fail(UPH_IO_ERROR, "uph_write_output: writing the diagnostics files in " + dir + " failed");
  return UPH_OK;
}
