// Leapfrog kick-drift of src/bin/sph.cc:90-168, one thread per fluid slot,
// with the reference's operation order so the state matches it bit for bit
// whenever the rates do.  Also the wall motion of inputbp.c:194-207 and the
// per-particle quantities the rate pass reads.
#include "uph_internal.cuh"

namespace uph {

// sph.cc:93-125 (itime != 1): *_min <- current, local* <- current, then the
// half kick with the predictor rates and the fluctuations of the previous
// rate evaluation.
__global__ void k_predict(const DevParams P, const SlotArrays S)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const double dt = P.dt;
  const double rho = S.rho[a], p = S.p[a], u = S.u[a], v = S.v[a];
  const double drho_a = S.drho_a[a], dp_a = S.dp_a[a];
  S.rho_min[a] = rho;
  S.p_min[a] = p;
  S.rho[a] = rho + 0.5 * dt * drho_a;
  S.rhot[a] = rho + 0.5 * dt * drho_a + S.frho[a];
  S.p[a] = p + 0.5 * dt * dp_a;
  S.pt[a] = p + 0.5 * dt * dp_a + S.fp[a];
  S.u_min[a] = u;
  S.v_min[a] = v;
  const double ax_a = S.ax_a[a], ay_a = S.ay_a[a];
  const double un = u + 0.5 * dt * ax_a, vn = v + 0.5 * dt * ay_a;
  S.u[a] = un;
  S.v[a] = vn;
  S.ut[a] = un + 0.5 * dt * ax_a + P.eps * S.fu[a];
  S.vt[a] = vn + 0.5 * dt * ay_a + P.eps * S.fv[a];
}

void launch_predict(const DevParams &P, const SlotArrays &S, cudaStream_t s)
{
  if (P.nf > 0) k_predict<<<(P.nf + 255) / 256, 256, 0, s>>>(P, S);
}

// sph.cc:137-168: the corrector with the rates just evaluated, then the
// drift x += dt v.  Flags non-finite results.
__global__ void k_correct(const DevParams P, const SlotArrays S, int first_step, unsigned *err)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const double dt = P.dt;
  const double drho = S.drho[a], dp = S.dp[a], ax = S.ax[a], ay = S.ay[a];
  const double frho = S.frho[a], fp = S.fp[a], fu = P.eps * S.fu[a], fv = P.eps * S.fv[a];
  double rho, p, u, v;
  if (first_step) {
    const double rho0 = S.rho[a], p0 = S.p[a], u0 = S.u[a], v0 = S.v[a];
    S.rhot[a] = rho0 + 0.5 * dt * drho + frho;
    rho = rho0 + 0.5 * dt * drho;
    S.pt[a] = p0 + 0.5 * dt * dp + fp;
    p = p0 + 0.5 * dt * dp;
    S.ut[a] = u0 + 0.5 * dt * ax + fu;
    S.vt[a] = v0 + 0.5 * dt * ay + fv;
    u = u0 + 0.5 * dt * ax;
    v = v0 + 0.5 * dt * ay;
  } else {
    const double rmin = S.rho_min[a], pmin = S.p_min[a], umin = S.u_min[a], vmin = S.v_min[a];
    S.rhot[a] = rmin + dt * drho + frho;
    rho = rmin + dt * drho;
    S.pt[a] = pmin + dt * dp + fp;
    p = pmin + dt * dp;
    S.ut[a] = umin + dt * ax + fu;
    S.vt[a] = vmin + dt * ay + fv;
    u = umin + dt * ax;
    v = vmin + dt * ay;
  }
  if (P.profile == UPH_PROFILE_WCSPH) {
    // the WCSPH pressure is the algebraic Tait law of the new density
    p = P.B * (pow(rho / P.rho0, P.gamma) - 1.0);
    S.pressure[a] = p;
  }
  S.rho[a] = rho;
  S.p[a] = p;
  S.u[a] = u;
  S.v[a] = v;
  const double x = S.x[a] + dt * u, y = S.y[a] + dt * v;
  S.x[a] = x;
  S.y[a] = y;
  if (!isfinite(rho) || !isfinite(p) || !isfinite(x) || !isfinite(y) || !isfinite(u) || !isfinite(v))
    atomicOr(err, ERR_NAN);
}

void launch_correct(const DevParams &P, const SlotArrays &S, int first_step, unsigned *err, cudaStream_t s)
{
  if (P.nf > 0) k_correct<<<(P.nf + 255) / 256, 256, 0, s>>>(P, S, first_step, err);
}

// 1/rho and 1/rhot for the rate pass; for WCSPH also p = B((rho/rho0)^g - 1)
// (derivatives.c:1674-1682) since that profile's pressure is a function of
// the density.
__global__ void k_refresh(const DevParams P, const SlotArrays S, int first, int count)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int a = first + k;
  const double rho = S.rho[a];
  S.inv_rho[a] = 1.0 / rho;
  S.inv_rhot[a] = 1.0 / S.rhot[a];
  if (P.profile == UPH_PROFILE_WCSPH) {
    const double pr = P.B * (pow(rho / P.rho0, P.gamma) - 1.0);
    S.p[a] = pr;
    S.pressure[a] = pr;
  }
}

void launch_refresh_inverse(const DevParams &P, const SlotArrays &S, int first, int count, cudaStream_t s)
{
  if (count > 0) k_refresh<<<(count + 255) / 256, 256, 0, s>>>(P, S, first, count);
}

// inputbp.c:194-207 (movingBoundary 1): the piston's particles all sit at
// x = S/2 (1 - cos wt) with u = ut = S w / 2 sin wt.  Slots of moving
// particles are found through their reference index.
__global__ void k_wall_motion(const DevParams P, const SlotArrays S, double t)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = P.nf + k;
  if (s >= P.n) return;
  const int o = S.orig[s];
  if (o < P.m0 || o >= P.b1) return;
  const double lbp = 0.5 * P.stroke * (1.0 - cos(P.omega * t));
  const double lbv = 0.5 * P.stroke * P.omega * sin(P.omega * t);
  S.x[s] = lbp;
  S.u[s] = lbv;
  S.ut[s] = lbv;
}

void launch_wall_motion(const DevParams &P, const SlotArrays &S, double t, cudaStream_t s)
{
  const int n = P.n - P.nf;
  if (n > 0) k_wall_motion<<<(n + 255) / 256, 256, 0, s>>>(P, S, t);
}

// EquationOfState for the non-fluid slots (derivatives.c:1674-1682); their
// density never changes, so once per upload is enough.
__global__ void k_wall_pressure(const DevParams P, const SlotArrays S)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = P.nf + k;
  if (s >= P.n) return;
  const double pr = P.B * (pow(S.rho[s] / P.rho0, P.gamma) - 1.0);
  S.pressure[s] = pr;
  if (P.profile == UPH_PROFILE_WCSPH) S.p[s] = pr;
}

void launch_wall_pressure(const DevParams &P, const SlotArrays &S, cudaStream_t s)
{
  const int n = P.n - P.nf;
  if (n > 0) k_wall_pressure<<<(n + 255) / 256, 256, 0, s>>>(P, S);
}

}  // namespace uph
