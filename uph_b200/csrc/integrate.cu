// Leapfrog kick-drift of src/bin/sph.cc:90-168, one thread per fluid slot,
// with the reference's operation order so the state matches it bit for bit
// whenever the rates do.  Also the wall motion of inputbp.c:194-207 and the
// per-particle quantities the rate pass reads.
//
// Inside a multi-step call the corrector of step n and the predictor of step
// n + 1 run in one kernel (they touch the same per-particle state and the
// predictor needs nothing the corrector does not already hold); the first
// step of a call uses the stand-alone predictor.
#include <algorithm>

#include "uph_internal.cuh"

namespace uph {

// WCSPH pressure is the algebraic Tait law of the density (derivatives.c:1674-1682)
__device__ __forceinline__ double tait(const DevParams &P, double rho)
{
  return P.B * (pow(rho / P.rho0, P.gamma) - 1.0);
}

// the FP32-pair pass's per-particle operands, rounded once from FP64
__device__ __forceinline__ void store_pair_operands(const SlotArrays &S, int a, double m, double p, double inv_rho,
                                                    double rho)
{
  S.pk[a] = make_float4((float)m, (float)(p * inv_rho * inv_rho), (float)rho, 0.0f);
}

// sph.cc:93-125 (itime != 1) for one particle whose post-step state is
// (rho, p, u, v): *_min <- current, local* <- current, then the half kick
// with the predictor rates and the fluctuations of the last rate
// evaluation.  Also refreshes 1/rho and 1/rhot for the next rate pass.
__device__ __forceinline__ void predict_one(const DevParams &P, const SlotArrays &S, int a, double rho, double p,
                                            double u, double v)
{
  const double dt = P.dt;
  const double drho_a = S.drho_a[a], dp_a = S.dp_a[a];
  S.rho_min[a] = rho;
  S.p_min[a] = p;
  const double rn = rho + 0.5 * dt * drho_a;
  const double rt = rho + 0.5 * dt * drho_a + S.frho[a];
  double pn = p + 0.5 * dt * dp_a;
  S.pt[a] = p + 0.5 * dt * dp_a + S.fp[a];
  S.u_min[a] = u;
  S.v_min[a] = v;
  const double ax_a = S.ax_a[a], ay_a = S.ay_a[a];
  const double un = u + 0.5 * dt * ax_a, vn = v + 0.5 * dt * ay_a;
  S.u[a] = un;
  S.v[a] = vn;
  S.ut[a] = un + 0.5 * dt * ax_a + P.eps * S.fu[a];
  S.vt[a] = vn + 0.5 * dt * ay_a + P.eps * S.fv[a];
  if (P.profile == UPH_PROFILE_WCSPH) {
    pn = tait(P, rn);
    S.pressure[a] = pn;
  }
  S.rho[a] = rn;
  S.rhot[a] = rt;
  S.p[a] = pn;
  const double ir = 1.0 / rn;
  S.inv_rho[a] = ir;
  S.inv_rhot[a] = 1.0 / rt;
  if (P.precision == UPH_PREC_FP32_PAIR) store_pair_operands(S, a, S.m[a], pn, ir, rn);
}

__global__ void k_predict(const DevParams P, const SlotArrays S)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  predict_one(P, S, a, S.rho[a], S.p[a], S.u[a], S.v[a]);
}

void launch_predict(const DevParams &P, const SlotArrays &S, cudaStream_t s)
{
  if (P.nf > 0) k_predict<<<(P.nf + 255) / 256, 256, 0, s>>>(P, S);
}

// sph.cc:137-168: the corrector with the rates just evaluated, then the
// drift x += dt v.  With predict_next the predictor of the following step
// runs right after.  Flags non-finite results.
// A particle now at (x, y): raise the cell list's rebuild flag if it left
// its skin since the last build, and report it if it left the domain (the
// build, which also checks, may not run this step).
__device__ __forceinline__ void note_moved(const DevParams &P, int slot, double x, double y, unsigned *err)
{
  if (P.rebuild && (fabs(x - P.xbin[slot]) > P.skin || fabs(y - P.ybin[slot]) > P.skin)) atomicOr(P.rebuild, 1u);
  if (!(x >= P.lo_x && y >= P.lo_y && x <= P.hi_x && y <= P.hi_y)) atomicOr(err, ERR_OUT_OF_DOMAIN);
}

// Moving boundary particles (reference indices [m0, b1)), found through
// their slot's reference index.
//  - inputbp.c:194-207 (movingBoundary 1): the piston's particles all sit at
//    x = S/2 (1 - cos wt) with u = ut = S w / 2 sin wt;
//  - inputbp.c:209-223 (movingBoundary 3, the lid): x = x0 + U t,
//    u = ut = U, from each particle's base x0;
//  - inputbp.c:224-243 (movingBoundary 2, the gate): y = y0 + U t and
//    v = U while 0 < t < t_stop, else y = y0 + U t_stop and v = 0 (the
//    reference leaves the gate's local velocity alone);
//  - a WallTable shakes each particle about its own rest position with its
//    own half stroke and frequency (one entry per particle, e.g. every wall
//    of a sloshing tank moving rigidly).
__device__ __forceinline__ void wall_move_one(const DevParams &P, const SlotArrays &S, const WallTable &W, int s,
                                              double t, unsigned *err)
{
  const int o = S.orig[s];
  if (o < P.m0 || o >= P.b1) return;
  if (!W.enabled && P.moving_boundary == 3) {
    const double U = P.lid_velocity;
    const double x = U * t + W.base[o - P.m0];
    S.x[s] = x;
    S.u[s] = U;
    S.ut[s] = U;
    note_moved(P, s, x, S.y[s], err);
    return;
  }
  if (!W.enabled && P.moving_boundary == 2) {
    const double U = P.lid_velocity;
    double y;
    if (t > 0.0 && t < P.gate_stop) {
      y = U * t + W.base[o - P.m0];
      S.v[s] = U;
    } else {
      y = U * P.gate_stop + W.base[o - P.m0];
      S.v[s] = 0.0;
    }
    S.y[s] = y;
    note_moved(P, s, S.x[s], y, err);
    return;
  }
  double x, u;
  if (W.enabled) {
    const int m = o - P.m0;
    const double hs = W.hs[m], om = W.om[m];
    x = W.x0[m] + hs * (1.0 - cos(om * t));
    u = hs * om * sin(om * t);
  } else {
    x = 0.5 * P.stroke * (1.0 - cos(P.omega * t));
    u = 0.5 * P.stroke * P.omega * sin(P.omega * t);
  }
  S.x[s] = x;
  S.u[s] = u;
  S.ut[s] = u;
  note_moved(P, s, x, S.y[s], err);
}


// The corrector of the fluid slots; with predict_next also the next step's
// predictor, and with walls_next the next step's wall motion on the threads
// past the fluid (its time from the device step counter, which the next
// step's cell-list launch advances: (steps started + 1) dt).
__global__ void k_correct(const DevParams P, const SlotArrays S, const WallTable W, int first_step, int predict_next,
                          int walls_next, unsigned *err, const int *d_itime)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) {
    if (walls_next && a < P.n) wall_move_one(P, S, W, a, (*d_itime + 1) * P.dt, err);
    return;
  }
  const double dt = P.dt;
  const double drho = S.drho[a], dp = S.dp[a], ax = S.ax[a], ay = S.ay[a];
  const double frho = S.frho[a], fp = S.fp[a], fu = P.eps * S.fu[a], fv = P.eps * S.fv[a];
  double rho, p, u, v, rt, pt, ut, vt;
  if (first_step) {
    const double rho0 = S.rho[a], p0 = S.p[a], u0 = S.u[a], v0 = S.v[a];
    rt = rho0 + 0.5 * dt * drho + frho;
    rho = rho0 + 0.5 * dt * drho;
    pt = p0 + 0.5 * dt * dp + fp;
    p = p0 + 0.5 * dt * dp;
    ut = u0 + 0.5 * dt * ax + fu;
    vt = v0 + 0.5 * dt * ay + fv;
    u = u0 + 0.5 * dt * ax;
    v = v0 + 0.5 * dt * ay;
  } else {
    const double rmin = S.rho_min[a], pmin = S.p_min[a], umin = S.u_min[a], vmin = S.v_min[a];
    rt = rmin + dt * drho + frho;
    rho = rmin + dt * drho;
    pt = pmin + dt * dp + fp;
    p = pmin + dt * dp;
    ut = umin + dt * ax + fu;
    vt = vmin + dt * ay + fv;
    u = umin + dt * ax;
    v = vmin + dt * ay;
  }
  if (P.profile == UPH_PROFILE_WCSPH) {
    p = tait(P, rho);
    S.pressure[a] = p;
  }
  const double x = S.x[a] + dt * u, y = S.y[a] + dt * v;
  S.x[a] = x;
  S.y[a] = y;
  if (!isfinite(rho) || !isfinite(p) || !isfinite(x) || !isfinite(y) || !isfinite(u) || !isfinite(v))
    atomicOr(err, ERR_NAN);
  note_moved(P, a, x, y, err);
  if (predict_next) {
    predict_one(P, S, a, rho, p, u, v);
  } else {
    S.rho[a] = rho;
    S.p[a] = p;
    S.u[a] = u;
    S.v[a] = v;
    S.rhot[a] = rt;
    S.pt[a] = pt;
    S.ut[a] = ut;
    S.vt[a] = vt;
  }
}

void launch_correct(const DevParams &P, const SlotArrays &S, const WallTable &W, int first_step, int predict_next,
                    int walls_next, unsigned *err, const int *d_itime, cudaStream_t s)
{
  const int n = std::max(walls_next ? P.n : P.nf, 1);
  k_correct<<<(n + 255) / 256, 256, 0, s>>>(P, S, W, first_step, predict_next, walls_next, err, d_itime);
}

// 1/rho and 1/rhot for the rate pass; for WCSPH also the Tait pressure; for
// FP32 pair arithmetic the packed operands.
// Needed where no predictor ran: a fresh upload and the first step.
__global__ void k_refresh(const DevParams P, const SlotArrays S, int first, int count)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int a = first + k;
  const double rho = S.rho[a];
  const double ir = 1.0 / rho;
  S.inv_rho[a] = ir;
  S.inv_rhot[a] = 1.0 / S.rhot[a];
  double pr = S.p[a];
  if (P.profile == UPH_PROFILE_WCSPH) {
    pr = tait(P, rho);
    S.p[a] = pr;
    S.pressure[a] = pr;
  }
  if (P.precision == UPH_PREC_FP32_PAIR) store_pair_operands(S, a, S.m[a], pr, ir, rho);
}

void launch_refresh_inverse(const DevParams &P, const SlotArrays &S, int first, int count, cudaStream_t s)
{
  if (count > 0) k_refresh<<<(count + 255) / 256, 256, 0, s>>>(P, S, first, count);
}

// the walls at the step's evaluation time: (steps started + 1) dt from the
// device step counter, else t_host
__global__ void k_wall_motion(const DevParams P, const SlotArrays S, const WallTable W, double t_host,
                              const int *d_itime, unsigned *err)
{
  const int s = P.nf + blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.n) return;
  wall_move_one(P, S, W, s, d_itime ? (*d_itime + 1) * P.dt : t_host, err);
}

void launch_wall_motion(const DevParams &P, const SlotArrays &S, const WallTable &W, double t_host,
                        const int *d_itime, unsigned *err, cudaStream_t s)
{
  const int n = P.n - P.nf;
  if (n > 0) k_wall_motion<<<(n + 255) / 256, 256, 0, s>>>(P, S, W, t_host, d_itime, err);
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
