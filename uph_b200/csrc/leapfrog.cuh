// The leapfrog corrector and predictor of src/bin/sph.cc:90-168 for one
// fluid particle, the WCSPH profile's algebraic Tait pressure and the wall
// laws of inputbp.c:194-243, shared by the stand-alone corrector
// (integrate.cu) and the rate passes that apply the step in their epilogue
// (ref_pass.cu, wcsph_pass.cu).
//
// Every sum and product is an explicitly rounded intrinsic (__dadd_rn,
// __dsub_rn, __dmul_rn, __ddiv_rn) in the reference's evaluation order, so
// the results are the same bits whatever the including file's multiply-add
// contraction setting, and equal to the reference's own (compiled without
// contraction) whenever the rates are.  (cos, sin and pow return the same
// bits with and without contraction.)
#pragma once

#include "uph_internal.cuh"

namespace uph {

// The rates the corrector reads, as the rate pass leaves them (fu, fv before
// the factor epsilon).
struct LeapRates {
  double drho, dp, ax, ay;  // ddensitydt, dpdt, dvdt
  double frho, fp, fu, fv;  // density / pressure / velocity fluctuation
};

// One particle's state after a corrector, and its local* fields.
struct LeapState {
  double rho, p, u, v;
  double rt, pt, ut, vt;
};

// sph.cc:137-168 (the correction after derivatives()): from the base state
// (the current state on the first step, with half a step, else the *_min
// state with a whole step),
//   rho = base + k drho,   rhot = (base + k drho) + frho,  likewise p,
//   u = base + k ax,       ut = (base + k ax) + eps fu,    likewise v.
__device__ __forceinline__ LeapState leap_correct(double dt, double eps, bool first, double rho0, double p0, double u0,
                                                  double v0, const LeapRates &R)
{
  const double k = first ? __dmul_rn(0.5, dt) : dt;
  LeapState o;
  o.rho = __dadd_rn(rho0, __dmul_rn(k, R.drho));
  o.rt = __dadd_rn(o.rho, R.frho);
  o.p = __dadd_rn(p0, __dmul_rn(k, R.dp));
  o.pt = __dadd_rn(o.p, R.fp);
  o.u = __dadd_rn(u0, __dmul_rn(k, R.ax));
  o.ut = __dadd_rn(o.u, __dmul_rn(eps, R.fu));
  o.v = __dadd_rn(v0, __dmul_rn(k, R.ay));
  o.vt = __dadd_rn(o.v, __dmul_rn(eps, R.fv));
  return o;
}

// the drift x + dt u
__device__ __forceinline__ double leap_drift(double dt, double x, double u) { return __dadd_rn(x, __dmul_rn(dt, u)); }

// sph.cc:93-125 (the prediction before derivatives(), itime != 1) for a
// particle whose post-step state is (rho, p, u, v): half a kick with the
// predictor rates of the last rate evaluation,
//   rho' = rho + dt/2 drho_a,  rhot' = rho' + frho,  likewise p,
//   u' = u + dt/2 ax_a,        ut' = (u' + dt/2 ax_a) + eps fu,  likewise v.
// *_min take the post-step state.
struct LeapPred {
  double rho, p, u, v, rt, pt, ut, vt;
  double ir, irt;  // 1 / rho', 1 / rhot' for the next rate pass
};
__device__ __forceinline__ LeapPred leap_predict(double dt, double eps, double rho, double p, double u, double v,
                                                 double drho_a, double dp_a, double ax_a, double ay_a, double frho,
                                                 double fp, double fu, double fv)
{
  const double hdt = __dmul_rn(0.5, dt);
  LeapPred o;
  o.rho = __dadd_rn(rho, __dmul_rn(hdt, drho_a));
  o.rt = __dadd_rn(o.rho, frho);
  o.p = __dadd_rn(p, __dmul_rn(hdt, dp_a));
  o.pt = __dadd_rn(o.p, fp);
  o.u = __dadd_rn(u, __dmul_rn(hdt, ax_a));
  o.v = __dadd_rn(v, __dmul_rn(hdt, ay_a));
  o.ut = __dadd_rn(__dadd_rn(o.u, __dmul_rn(hdt, ax_a)), __dmul_rn(eps, fu));
  o.vt = __dadd_rn(__dadd_rn(o.v, __dmul_rn(hdt, ay_a)), __dmul_rn(eps, fv));
  o.ir = __ddiv_rn(1.0, o.rho);
  o.irt = __ddiv_rn(1.0, o.rt);
  return o;
}

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
    const double x = __dadd_rn(__dmul_rn(U, t), W.base[o - P.m0]);
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
      y = __dadd_rn(__dmul_rn(U, t), W.base[o - P.m0]);
      S.v[s] = U;
    } else {
      y = __dadd_rn(__dmul_rn(U, P.gate_stop), W.base[o - P.m0]);
      S.v[s] = 0.0;
    }
    S.y[s] = y;
    note_moved(P, s, S.x[s], y, err);
    return;
  }
  double x, u;
  if (W.enabled) {
    // x0 + hs (1 - cos wt), hs w sin wt
    const int m = o - P.m0;
    const double hs = W.hs[m], om = W.om[m];
    const double ph = __dmul_rn(om, t);
    x = __dadd_rn(W.x0[m], __dmul_rn(hs, __dsub_rn(1.0, cos(ph))));
    u = __dmul_rn(__dmul_rn(hs, om), sin(ph));
  } else {
    // S/2 (1 - cos wt), S/2 w sin wt
    const double hs = __dmul_rn(0.5, P.stroke);
    const double ph = __dmul_rn(P.omega, t);
    x = __dmul_rn(hs, __dsub_rn(1.0, cos(ph)));
    u = __dmul_rn(__dmul_rn(hs, P.omega), sin(ph));
  }
  S.x[s] = x;
  S.u[s] = u;
  S.ut[s] = u;
  note_moved(P, s, x, S.y[s], err);
}

// WCSPH pressure is the algebraic Tait law of the density (derivatives.c:1674-1682)
__device__ __forceinline__ double tait(const DevParams &P, double rho)
{
  return __dmul_rn(P.B, __dsub_rn(pow(__ddiv_rn(rho, P.rho0), P.gamma), 1.0));
}

}  // namespace uph
