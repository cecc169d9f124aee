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

#include "leapfrog.cuh"

namespace uph {

// sph.cc:93-125 (itime != 1) for one particle whose post-step state is
// (rho, p, u, v): *_min <- current, local* <- current, then the half kick
// with the predictor rates and the fluctuations of the last rate
// evaluation (leap_predict).  Also refreshes 1/rho and 1/rhot for the next
// rate pass.
__device__ __forceinline__ void predict_one(const DevParams &P, const SlotArrays &S, int a, double rho, double p,
                                            double u, double v)
{
  const LeapPred q = leap_predict(P.dt, P.eps, rho, p, u, v, S.drho_a[a], S.dp_a[a], S.ax_a[a], S.ay_a[a], S.frho[a],
                                  S.fp[a], S.fu[a], S.fv[a]);
  S.rho_min[a] = rho;
  S.p_min[a] = p;
  S.u_min[a] = u;
  S.v_min[a] = v;
  S.u[a] = q.u;
  S.v[a] = q.v;
  S.ut[a] = q.ut;
  S.vt[a] = q.vt;
  S.pt[a] = q.pt;
  double pn = q.p;
  if (P.profile == UPH_PROFILE_WCSPH) {
    pn = tait(P, q.rho);
    S.pressure[a] = pn;
  }
  S.rho[a] = q.rho;
  S.rhot[a] = q.rt;
  S.p[a] = pn;
  S.inv_rho[a] = q.ir;
  S.inv_rhot[a] = q.irt;
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
  const LeapRates R = {S.drho[a], S.dp[a], S.ax[a], S.ay[a], S.frho[a], S.fp[a], S.fu[a], S.fv[a]};
  const LeapState c = first_step ? leap_correct(P.dt, P.eps, true, S.rho[a], S.p[a], S.u[a], S.v[a], R)
                                 : leap_correct(P.dt, P.eps, false, S.rho_min[a], S.p_min[a], S.u_min[a], S.v_min[a], R);
  const double rho = c.rho, u = c.u, v = c.v, rt = c.rt, pt = c.pt, ut = c.ut, vt = c.vt;
  double p = c.p;
  if (P.profile == UPH_PROFILE_WCSPH) {
    p = tait(P, rho);
    S.pressure[a] = p;
  }
  const double x = leap_drift(P.dt, S.x[a], u), y = leap_drift(P.dt, S.y[a], v);
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

// 1/rho and 1/rhot for the rate pass; for WCSPH also the Tait pressure.
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
