// The fused rate pass of the REF profile: one thread per fluid particle
// gathers every pair term of the reference's derivatives() from the cells
// within `reach` cells of its own (5 x 5 cells of half the radius by
// default), in FP64.
//
// The reference evaluates each term as a scatter loop over pairs (i < j)
// that adds one formula to i and another to j.  Here particle a sees every
// neighbour b; a plays the reference's i when orig(a) < orig(b) and its j
// otherwise.  With g = F(r) (x_a - x_b) (= the reference's dwcdx for the
// pair when a is i, and its negation when a is j), the per-a contributions
// are (V = m / rho, P = rho0 c0^2 + gamma p, ms = m_b if a is i else m_a):
//
//   ddensitydt_approx  (PredictingDensityEquation, derivatives.c:1217-1252)
//       i: m_b (v_a - vt_b).g        j: m_a (vt_a - v_b).g
//   dpdt_approx        (PredictingDynamicPressureEquation, :1254-1331)
//       m_b/rho_a P_a (v_a - v_b).g + gamma kappa ms/rho_b (p_a - p_b) nu 4P_a/(P_a+P_b)
//       - kappa P_a ms/rho_b (rho_a - rho_b)(1/rho_a + 1/rho_b) nu
//   dvdt_approx        (PredictingPressureGradientForce, :1333-1377)
//       -m_b (p_a/rho_a^2 + p_b/rho_b^2) g
//   densityFluctuation / pressureFluctuation (:2100-2172)
//       -V_b (f_a - f_b) W
//   velocityFluctuation (:2060-2097), i side only
//       (v_a - v_b) W (m_a/rhot_b - m_b/rhot_a)
//   ddensitydt         (DensityEquation, :1520-1567)
//       V_b rhot_b (v_a - vt_b).g
//   dpdt               (DynamicPressureEquation, :1569-1672)
//       V_b rhot_b/rho_a P_a (v_a - vt_b).g + gamma kappa V_b (p_a - pt_b) nu 4P_a/(P_a+P_b)
//       - kappa P_a V_b (rho_a - rhot_b)(1/rho_a + 1/rho_b) nu
//   dvdt               (PressureGradientForce, :1109-1163)
//       -m_b (p_a rhot_b/(rho_a^2 rho_b) + p_b rhot_a/(rho_b^2 rho_a)) g
//   dvdt viscous       (ViscousForcesSingleStep, :1770-1839)
//       s m_b mu_ab/(r^2 + 0.01h^2) (rhot_b/(rho_a^2 rho_b) - rhot_a/(rho_b^2 rho_a)) S.g,
//       s = +1 on the i side and -1 on the j side (the reference's jSigma is
//       -iSigma, so the pair force is a difference, not a sum)
//   dvdt_approx viscous (PredictingViscousForcesSingleStep, :1448-1515)
//       m_b mu_ab/(r^2 + 0.01h^2) (1/rho_a^2 + 1/rho_b^2) S.g
//   with nu = (x_a - x_b).g / (r^2 + 0.01 h^2), mu_ab = 2 mu rho_a rho_b/(rho_a + rho_b),
//   S = [[s00, s01], [s01, -s00]], s00 = dx' du - dy' dv, s01 = dx' dv + dy' du,
//   (dx', dy') = x_b - x_a, (du, dv) = v_a - v_b.
// Wall forces (derivatives.c:2396-2449, 1392-1446 and the other modes),
// gravity (:1167-1178, 1379-1390), the sponge layer (:2827-2838) and the
// algebraic Tait pressure (:1674-1682) are added in the same pass.
//
// A pair exists iff it would be in the reference's list: both particles
// interacting, max(orig a, orig b) < ParticleBoundary (Search.cc:33 with
// derivatives.c:1082-1084), DBL_EPSILON < r^2 < (h h) 4 where r^2 is
// dx*dx + dy*dy rounded exactly like the reference (no fused multiply-add).
//
// Execution: one CTA per storage tile of T x T cells (tile_pass.cuh).  The
// CTA stages the records of its tile and of the `reach` cells around it in
// shared memory, once; each thread then owns one fluid particle of the tile.
// Per particle, a cheap listing phase walks its (2 reach + 1)^2 stencil in
// shared memory with only the exact distance test and lists the in-radius
// partners; then the warp runs the FP64 pair arithmetic over those lists,
// which have nearly equal lengths, so the lanes of a warp stay converged in
// the expensive loop.
#include <limits.h>

#include "leapfrog.cuh"
#include "tile_pass.cuh"

namespace uph {

struct RefAcc {
  double drho, dp, ax, ay;
  double drho_a, dp_a, ax_a, ay_a;
  double frho, fp, fu, fv;
};

// wall forces of a listed pair whose i side is this fluid particle
__device__ __forceinline__ void wall_pair_force(const DevParams &P, int itb, double r2, double dxa, double dya,
                                                double dua, double dva, double ma, RefAcc &A)
{
  const double r = sqrt(r2);
  double sx = 0.0, sy = 0.0;
  // SpringBoundaryForces / PredictingSpringBoundaryForces (derivatives.c:2396-2449, 1392-1446)
  if (itb == 2 || itb == 3 || itb == 5) {
    const double r0 = 3.0 * P.dx;
    if (r < r0) {
      const double rv = dxa * dua + dya * dva;
      const double c1 = P.k_spring * (r0 - r) / (r * ma);
      const double c2 = P.c_damp * rv / (r * r * ma);
      sx = -c1 * dxa - c2 * dxa;
      sy = -c1 * dya - c2 * dya;
    }
  }
  A.ax_a += sx;
  A.ay_a += sy;
  if (P.boundary_force == 3) {
    A.ax += sx;
    A.ay += sy;
  } else if (P.boundary_force == 4 && (itb == 2 || itb == 3) && r < P.dx) {
    // ImprovedMonaghan, derivatives.c:1955-2012
    const double hh = P.h;
    const double norm = 7.0 / (64.0 * 3.142 * hh * hh);
    const double q = r / hh;
    double phi = 0.0;
    if (q < 2.0) {
      const double t = 2.0 - q;
      phi = norm * (1.0 + 2.0 * q) * (t * t) * (t * t);
    }
    const double rd = r - P.dx / 5.0;
    const double vmax = P.mach_c * P.mach_c / 5.0;
    const double c = vmax * phi / (rd * r);
    A.ax += c * dxa;
    A.ay += c * dya;
  } else if (P.boundary_force == 5 && itb == 2 && r < P.dx) {
    // SerialSpringBoundaryForces, derivatives.c:2452-2479
    A.ax -= (P.k_spring * dxa + P.c_damp * dua) / ma;
    A.ay -= (P.k_spring * dya + P.c_damp * dva) / ma;
  }
}

// ---- partner records -----------------------------------------------------------
// One particle's fields as the pair loop reads them: the SoA state plus the
// per-particle factors every pair would otherwise recompute (Tait's
// rho0 c0^2 + gamma p, 1/rho^2, rhot/rho, m/rho).  144 bytes, read as nine
// 16-byte shared-memory loads.
// (The listing's FP32 positions, relative to the CTA's block origin, are a
// separate shared-memory array: the pair loop never reads them.)
struct __align__(16) RefRec {
  double x, y, u, v, ut, vt, rho, rhot, p, pt, m, ir, irt, P, ir2, C, V;
  int orig, itype;
};
static_assert(sizeof(RefRec) == 144, "RefRec is nine 16-byte chunks");

__device__ __forceinline__ RefRec load_ref_rec(const DevParams &P, const SlotArrays &S, int s)
{
  RefRec r;
  r.x = S.x[s];
  r.y = S.y[s];
  r.u = S.u[s];
  r.v = S.v[s];
  r.ut = S.ut[s];
  r.vt = S.vt[s];
  r.rho = S.rho[s];
  r.rhot = S.rhot[s];
  r.p = S.p[s];
  r.pt = S.pt[s];
  r.m = S.m[s];
  r.ir = S.inv_rho[s];
  r.irt = S.inv_rhot[s];
  r.P = fma(P.gamma, r.p, P.rho0c2);
  r.ir2 = r.ir * r.ir;
  r.C = r.rhot * r.ir;
  r.V = r.m * r.ir;
  r.orig = S.orig[s];
  r.itype = S.itype[s];
  return r;
}

// The particle a thread owns, with its per-particle constants.
struct RefOwn {
  RefRec r;
  double IPa;  // P_a / rho_a
  double G4a;  // 4 gamma kappa P_a
  double KPa;  // kappa P_a
  double A1a;  // p_a / rho_a^2
};

__device__ __forceinline__ RefOwn make_own(const DevParams &P, const RefRec &r)
{
  RefOwn o;
  o.r = r;
  o.IPa = r.ir * r.P;
  o.G4a = 4.0 * (P.gamma * P.kappa) * r.P;
  o.KPa = P.kappa * r.P;
  o.A1a = r.p * r.ir2;
  return o;
}

// The per-a sums of one pair (a, b), a = the own particle.  With
// g = F (x_a - x_b) and the header's formulas, rearranged so that the pair
// shares one reciprocal and per-particle factors come from the records:
//   1 / (r^2 + 0.01 h^2), 1 / (P_a + P_b) and 1 / (1/rho_a + 1/rho_b)
//   all from rr = 1 / ((r^2 + 0.01 h^2)(P_a + P_b)(1/rho_a + 1/rho_b));
//   (x_a - x_b) . g = F r^2;
//   S . g = -F r^2 (v_a - v_b) for the deviatoric S of the viscous terms
//   (its terms in dx dy dv cancel exactly), so both viscous forces are
//   multiples of (v_a - v_b).
__device__ __forceinline__ void ref_pair(const DevParams &P, const RefOwn &a, const RefRec &b, bool isI, RefAcc &A)
{
  const double dxa = a.r.x - b.x, dya = a.r.y - b.y;
  const double r2 = exact_r2(dxa, dya);
  // poly-7 convolution W and deconvolution gradient factor, functions of q^2
  const double q2 = r2 * P.inv_h2;
  const double t = fma(-0.25, q2, 1.0);
  const double t2 = t * t, t4 = t2 * t2;
  const double t7 = t4 * t2 * t, t8 = t4 * t4;
  const double pp = fma(fma(fma(fma(fma(fma(305.0, q2, -628.0), q2, 1184.0), q2, -1984.0), q2, 2816.0), q2, -3072.0), q2, 2048.0);
  const double pp7 = fma(fma(fma(fma(fma(fma(305.0, q2, -1106.0), q2, 1912.0), q2, -2912.0), q2, 3712.0), q2, -3584.0), q2, 2048.0);
  const double W = P.w_alpha * t8 * pp;
  const double F = P.dw_alpha_h2 * t7 * pp7;
  const double Fr2 = F * r2;

  const double De = r2 + P.eta2;
  const double SP = a.r.P + b.P;
  const double Sr = a.r.ir + b.ir;
  const double SPSr = SP * Sr;
  const double rr = rcp_nr(De * SPSr);
  const double inv_r2e = rr * SPSr;
  const double invSP = rr * (De * Sr);
  const double nu = Fr2 * inv_r2e;

  const double dux = a.r.u - b.u, duy = a.r.v - b.v;
  const double eux = a.r.u - b.ut, euy = a.r.v - b.vt;
  const double Vd = fma(dux, dxa, duy * dya);
  const double Ed = fma(eux, dxa, euy * dya);
  const double pdx = isI ? eux : a.r.ut - b.u;
  const double pdy = isI ? euy : a.r.vt - b.v;
  const double Pd = fma(pdx, dxa, pdy * dya);
  const double ms = isI ? b.m : a.r.m;
  const double mbF = b.m * F;

  // predictor density (PredictingDensityEquation)
  A.drho_a = fma(ms * F, Pd, A.drho_a);
  // predictor pressure (PredictingDynamicPressureEquation)
  const double dpp = a.r.p - b.p, dr = a.r.rho - b.rho;
  const double brk = fma(-(a.KPa * dr), Sr, a.G4a * dpp * invSP);
  A.dp_a = fma(mbF * a.IPa, Vd, A.dp_a);
  A.dp_a = fma(ms * b.ir * nu, brk, A.dp_a);
  // fluctuations
  const double VW = b.V * W;
  A.frho = fma(-VW, dr, A.frho);
  A.fp = fma(-VW, dpp, A.fp);
  const double cfv = isI ? fma(a.r.m, b.irt, -(b.m * a.r.irt)) * W : 0.0;
  A.fu = fma(dux, cfv, A.fu);
  A.fv = fma(duy, cfv, A.fv);
  // continuity (DensityEquation)
  const double VrF = b.V * b.rhot * F;
  A.drho = fma(VrF, Ed, A.drho);
  // rate-form Tait with diffusion (DynamicPressureEquation)
  const double dpt = a.r.p - b.pt, drt = a.r.rho - b.rhot;
  const double brk2 = fma(-(a.KPa * drt), Sr, a.G4a * dpt * invSP);
  A.dp = fma(VrF * a.IPa, Ed, A.dp);
  A.dp = fma(b.V * nu, brk2, A.dp);
  // pressure gradients (PredictingPressureGradientForce, PressureGradientForce)
  const double A1b = b.p * b.ir2;
  const double c1 = mbF * (a.A1a + A1b);
  const double c2 = mbF * fma(a.A1a, b.C, A1b * a.r.C);
  A.ax_a = fma(-c1, dxa, A.ax_a);
  A.ay_a = fma(-c1, dya, A.ay_a);
  A.ax = fma(-c2, dxa, A.ax);
  A.ay = fma(-c2, dya, A.ay);
  // deviatoric viscous stress (ViscousForcesSingleStep and its predictor):
  // m_b mu_ab / (r^2 + 0.01 h^2) times F r^2 = m_b 2 mu rr (P_a + P_b) F r^2
  // stressType 2 keeps the single-step predictor; its corrector force is
  // added after the pass (launch_viscous_two_step)
  if (P.stress_type == 1 || P.stress_type == 2) {
    const double vis = b.m * P.two_mu0 * rr * SP * Fr2;
    const double vp = vis * (a.r.ir2 + b.ir2);
    A.ax_a = fma(-vp, dux, A.ax_a);
    A.ay_a = fma(-vp, duy, A.ay_a);
    if (P.stress_type == 1) {
      const double D = fma(b.C, a.r.ir2, -(a.r.C * b.ir2));
      const double sv = (isI ? vis : -vis) * D;
      A.ax = fma(-sv, dux, A.ax);
      A.ay = fma(-sv, duy, A.ay);
    }
  }
  // wall forces: only pairs whose i is this fluid particle
  if (isI && a.r.itype == 1 && b.itype >= 2) wall_pair_force(P, b.itype, r2, dxa, dya, dux, duy, a.r.m, A);
}

// gravity, sponge, Tait pressure, stores
__device__ __forceinline__ void ref_epilogue(const DevParams &P, const SlotArrays &S, int a, const RefOwn &o,
                                             RefAcc &A, double bx, double by)
{
  A.ax += bx;
  A.ay += by;
  if (P.gravity_flag == 1) {
    A.ay -= P.g;
    A.ay_a -= P.g;
  }
  if (P.moving_boundary == 1 && P.wave_absorption == 1) A.ax -= S.sponge[a] * o.r.u;
  S.drho[a] = A.drho;
  S.dp[a] = A.dp;
  S.ax[a] = A.ax;
  S.ay[a] = A.ay;
  S.drho_a[a] = A.drho_a;
  S.dp_a[a] = A.dp_a;
  S.ax_a[a] = A.ax_a;
  S.ay_a[a] = A.ay_a;
  S.frho[a] = A.frho;
  S.fp[a] = A.fp;
  S.fu[a] = A.fu;
  S.fv[a] = A.fv;
  S.pressure[a] = P.B * (pow(o.r.rho / P.rho0, P.gamma) - 1.0);
}

// The epilogue of a pass that applies the step (StepOut): the same rates as
// ref_epilogue, then the corrector with them, the drift and, with
// predict_next, the next step's predictor (sph.cc:93-168, leapfrog.cuh),
// all written to slot a of the other buffer.  The rates and the algebraic
// pressure are stored only by the last step of a call (no predictor
// follows): inside a call nothing reads them before that step writes them
// again, and the step's own predictor has used them already.  The
// particle's constants (mass, type, reference index, sponge factor) are the
// same in both buffers and are not written.  S is only read here, at the
// particle's own slot.
__device__ __forceinline__ void ref_step_epilogue(const DevParams &P, const SlotArrays &S, const StepOut &F, int a,
                                                  const RefOwn &o, RefAcc &A, double bx, double by)
{
  const SlotArrays &D = F.D;
  A.ax += bx;
  A.ay += by;
  if (P.gravity_flag == 1) {
    A.ay -= P.g;
    A.ay_a -= P.g;
  }
  if (P.moving_boundary == 1 && P.wave_absorption == 1) A.ax -= S.sponge[a] * o.r.u;
  if (!F.predict_next) {
    D.drho[a] = A.drho;
    D.dp[a] = A.dp;
    D.ax[a] = A.ax;
    D.ay[a] = A.ay;
    D.drho_a[a] = A.drho_a;
    D.dp_a[a] = A.dp_a;
    D.ax_a[a] = A.ax_a;
    D.ay_a[a] = A.ay_a;
    D.frho[a] = A.frho;
    D.fp[a] = A.fp;
    D.fu[a] = A.fu;
    D.fv[a] = A.fv;
    D.pressure[a] = P.B * (pow(o.r.rho / P.rho0, P.gamma) - 1.0);
  }
  const LeapRates R = {A.drho, A.dp, A.ax, A.ay, A.frho, A.fp, A.fu, A.fv};
  // the *_min state: the corrector's base after the first step, and carried
  // over unchanged when no predictor follows
  double rmin = 0.0, pmin = 0.0, umin = 0.0, vmin = 0.0;
  if (!F.first_step || !F.predict_next) {
    rmin = S.rho_min[a];
    pmin = S.p_min[a];
    umin = S.u_min[a];
    vmin = S.v_min[a];
  }
  const LeapState c = F.first_step ? leap_correct(P.dt, P.eps, true, o.r.rho, o.r.p, o.r.u, o.r.v, R)
                                   : leap_correct(P.dt, P.eps, false, rmin, pmin, umin, vmin, R);
  const double x = leap_drift(P.dt, o.r.x, c.u), y = leap_drift(P.dt, o.r.y, c.v);
  D.x[a] = x;
  D.y[a] = y;
  if (!isfinite(c.rho) || !isfinite(c.p) || !isfinite(x) || !isfinite(y) || !isfinite(c.u) || !isfinite(c.v))
    atomicOr(F.err, ERR_NAN);
  note_moved(P, a, x, y, F.err);
  if (F.predict_next) {
    const LeapPred q = leap_predict(P.dt, P.eps, c.rho, c.p, c.u, c.v, A.drho_a, A.dp_a, A.ax_a, A.ay_a, A.frho,
                                    A.fp, A.fu, A.fv);
    D.rho_min[a] = c.rho;
    D.p_min[a] = c.p;
    D.u_min[a] = c.u;
    D.v_min[a] = c.v;
    D.u[a] = q.u;
    D.v[a] = q.v;
    D.ut[a] = q.ut;
    D.vt[a] = q.vt;
    D.rho[a] = q.rho;
    D.rhot[a] = q.rt;
    D.p[a] = q.p;
    D.pt[a] = q.pt;
    D.inv_rho[a] = q.ir;
    D.inv_rhot[a] = q.irt;
  } else {
    D.rho_min[a] = rmin;
    D.p_min[a] = pmin;
    D.u_min[a] = umin;
    D.v_min[a] = vmin;
    D.u[a] = c.u;
    D.v[a] = c.v;
    D.ut[a] = c.ut;
    D.vt[a] = c.vt;
    D.rho[a] = c.rho;
    D.rhot[a] = c.rt;
    D.p[a] = c.p;
    D.pt[a] = c.pt;
    D.inv_rho[a] = __ddiv_rn(1.0, c.rho);
    D.inv_rhot[a] = __ddiv_rn(1.0, c.rt);
  }
}

// ---- the two partner sources ---------------------------------------------------------
// Staged: records in shared memory, list entries are record indices.
struct StagedSrc {
  const RefRec *rec;
  const float2 *posf;    // block-relative FP32 positions
  const double *cut_d2;  // the knn cap's cut per record (kKnn only)
  const int *cut_j;
  __device__ __forceinline__ double2 xy(int k) const { return *reinterpret_cast<const double2 *>(&rec[k].x); }
  __device__ __forceinline__ float2 xyf(int k) const { return posf[k]; }
  __device__ __forceinline__ int orig(int k) const { return rec[k].orig; }
  __device__ __forceinline__ double mass(int k) const { return rec[k].m; }
  __device__ __forceinline__ RefRec get(int k) const { return rec[k]; }
  __device__ __forceinline__ void cut(int k, double &d2, int &j) const
  {
    d2 = cut_d2[k];
    j = cut_j[k];
  }
};
// Global: the SoA arrays, list entries are slots.
struct GlobalSrc {
  DevParams P;
  SlotArrays S;
  __device__ __forceinline__ double2 xy(int s) const { return make_double2(S.x[s], S.y[s]); }
  __device__ __forceinline__ float2 xyf(int) const { return make_float2(0.f, 0.f); }  // not used: no pre-test
  __device__ __forceinline__ int orig(int s) const { return S.orig[s]; }
  __device__ __forceinline__ double mass(int s) const { return S.m[s]; }
  __device__ __forceinline__ RefRec get(int s) const { return load_ref_rec(P, S, s); }
  __device__ __forceinline__ void cut(int s, double &d2, int &j) const
  {
    d2 = P.kcut_d2[s];
    j = P.kcut_j[s];
  }
};
// Phase 1 and 2 for one own particle until its stencil is exhausted.
// nshort >= 0: the own particle's candidate list, nshort entries, is in its
// column of s_nb (kF32 only); else the stencil is walked, appending to
// vl_out (if not null) as tile_list does.
template <bool kBrute, bool kKnn, bool kF32, typename Src, typename Cursor, typename Entry>
__device__ __forceinline__ void ref_particle(const DevParams &P, const Src &src, Cursor &cur, bool active, int self,
                                             const RefOwn &o, const F32Test &ft, Entry *s_nb, RefAcc &A, double &bx,
                                             double &by, unsigned &my_pairs, int &my_nb, double cd, int cj,
                                             int nshort, unsigned short *vl_out, int &vl_cnt)
{
  constexpr Entry kRole = sizeof(Entry) == 2 ? (Entry)kRoleI16 : (Entry)kRoleI;
  const int col = threadIdx.x;
  bool more = active;
  while (__any_sync(0xffffffffu, more)) {
    int cnt = 0;
    if (kF32 && nshort >= 0) {
      if constexpr (kF32) {
        if (more)
          cnt = tile_list_short<kBrute, kKnn>(P, src, nshort, self, o.r.orig, o.r.x, o.r.y, ft, s_nb, col, my_pairs,
                                              my_nb, bx, by, cd, cj);
      }
      more = false;
    } else {
      cnt = tile_list<kBrute, kTileChunk, kKnn, kF32>(P, src, cur, more, self, o.r.orig, o.r.x, o.r.y, ft, s_nb, col,
                                                      my_pairs, my_nb, bx, by, cd, cj, vl_out, vl_cnt);
    }
    __syncwarp();
    for (int e = 0; e < cnt; e++) {
      const Entry ent = s_nb[e * kTileThreads + col];
      const RefRec b = src.get((int)(ent & (Entry)~kRole));
      ref_pair(P, o, b, (ent & kRole) != 0, A);
    }
    __syncwarp();
  }
}

// Dynamic shared memory of the tiled pass and its record capacity; with the
// knn cap every record also carries its query's cut (12 bytes).
template <bool kKnn>
__host__ __device__ constexpr int ref_rec_cap() { return kKnn ? 560 : 620; }
constexpr size_t kRefListBytes = sizeof(unsigned short) * kTileChunk * kTileThreads;
// per record: the record, its FP32 position and (kKnn) its cut
template <bool kKnn>
constexpr size_t ref_smem()
{
  return sizeof(TileBlock) + kRefListBytes + (sizeof(RefRec) + 8 + (kKnn ? 12 : 0)) * ref_rec_cap<kKnn>();
}
static_assert(sizeof(RefRec) * 560 >= sizeof(unsigned) * kTileChunk * kTileThreads,
              "the fallback's 32-bit lists live in the record area");

// One CTA per storage tile (see tile_pass.cuh).  Phase 1 lists in-radius
// partners per thread (the exact distance test only); phase 2 runs the FP64
// pair arithmetic over the lists, so the lanes of a warp stay converged in
// the expensive loop.
// kBrute: the wall modes that act on every boundary particle within the
// radius (LeonnardJonesBoundaryForces, MonaghanBoundaryForce) rather than on
// listed pairs.  kKnn: the reference's k-nearest cap (DevParams::knn).
// One tile (see tile_pass.cuh): stage the block's records, then each thread
// owns a fluid particle of the tile's core.  Phase 1 lists in-radius
// partners per thread (the exact distance test, after the FP32 pre-test);
// phase 2 runs the FP64 pair arithmetic over the lists, so the lanes of a
// warp stay converged in the expensive loop.
template <bool kBrute, bool kKnn>
__device__ __forceinline__ void ref_tile(const DevParams &P, const SlotArrays &S, const CellGrid &G,
                                         const StepOut &F, int tile, unsigned char *smem, unsigned &my_pairs,
                                         int &my_nb)
{
  constexpr int kCap = ref_rec_cap<kKnn>();
  TileBlock &B = *reinterpret_cast<TileBlock *>(smem);
  unsigned short *s_nb16 = reinterpret_cast<unsigned short *>(smem + sizeof(TileBlock));
  RefRec *rec = reinterpret_cast<RefRec *>(smem + sizeof(TileBlock) + kRefListBytes);
  float2 *s_posf = reinterpret_cast<float2 *>(rec + kCap);
  double *s_cd = reinterpret_cast<double *>(s_posf + kCap);
  int *s_cj = reinterpret_cast<int *>(s_cd + kCap);
  tile_setup(P, G, tile, B);
  const int ncore = B.ncore;
  if (ncore == 0) return;
  const bool staged = B.nrec <= kCap;
  // the origin of the block: the listing's FP32 positions are relative to it
  const double ox = P.lo_x + B.bx0 * P.cell, oy = P.lo_y + B.by0 * P.cell;
  if (staged) {
    // this tile's candidate lists are current if written since the last
    // build (G.vl null: the lists are off, every particle walks the stencil)
    const unsigned gen = G.vl ? *G.gen : 0u;
    const bool vl_use = G.vl && G.tile_gen[tile] == gen;
    // two records per thread at a time, every load issued before the first
    // store, so the staging waits for two rounds of loads (the slots, then
    // their fields) instead of two per record
    auto put = [&](int k, const RefRec &r, double cd, int cj) {
      rec[k] = r;
      s_posf[k] = make_float2((float)(r.x - ox), (float)(r.y - oy));
      if constexpr (kKnn) {
        s_cd[k] = cd;
        s_cj[k] = cj;
      }
    };
    for (int k0 = threadIdx.x; k0 < B.nrec; k0 += 2 * kTileThreads) {
      const int k1 = k0 + kTileThreads;
      const bool two = k1 < B.nrec;
      const int s0 = G.list[tile_record_pos(B, k0)];
      const int s1 = two ? G.list[tile_record_pos(B, k1)] : s0;
      // the candidate lists the core's fluid particles will read after the
      // staging: fetched into L2 meanwhile (the halo's too, for their tiles)
      if (vl_use) {
        if (s0 < P.nf) {
          prefetch_l2(G.vl + (size_t)s0 * kVlMax);
          prefetch_l2(G.vl_n + s0);
        }
        if (two && s1 < P.nf) {
          prefetch_l2(G.vl + (size_t)s1 * kVlMax);
          prefetch_l2(G.vl_n + s1);
        }
      }
      const RefRec r0 = load_ref_rec(P, S, s0);
      const RefRec r1 = load_ref_rec(P, S, s1);
      // only fluid queries have a cut; other records are never a pair's i
      // seen from a fluid particle that is its j
      double cd0 = 0.0, cd1 = 0.0;
      int cj0 = 0, cj1 = 0;
      if constexpr (kKnn) {
        if (s0 < P.nf) {
          cd0 = P.kcut_d2[s0];
          cj0 = P.kcut_j[s0];
        }
        if (s1 < P.nf) {
          cd1 = P.kcut_d2[s1];
          cj1 = P.kcut_j[s1];
        }
      }
      put(k0, r0, cd0, cj0);
      if (two) put(k1, r1, cd1, cj1);
    }
    __syncthreads();
    const StagedSrc src{rec, s_posf, s_cd, s_cj};
    for (int base = 0; base < ncore; base += kTileThreads) {
      const int k = base + threadIdx.x;
      int kr = 0, pos = 0, a = 0, cx = B.bx0, cy = B.by0;
      if (k < ncore) {
        tile_core_cell(B, k, kr, pos, cx, cy);
        a = G.list[pos];
      }
      const bool active = k < ncore && a < P.nf;
      // the epilogue's reads of the particle's own *_min state and sponge
      // factor: fetched into L2 now, while the pair loop runs
      if (F.enabled && active) {
        if (!F.first_step || !F.predict_next) {
          prefetch_l2(S.rho_min + a);
          prefetch_l2(S.p_min + a);
          prefetch_l2(S.u_min + a);
          prefetch_l2(S.v_min + a);
        }
        if (P.moving_boundary == 1 && P.wave_absorption == 1) prefetch_l2(S.sponge + a);
      }
      const RefOwn o = make_own(P, rec[active ? kr : 0]);
      StagedCursor cur;
      cur.c.init(B, P.reach, active ? cx : B.bx0, active ? cy : B.by0);
      double cd = 0.0;
      int cj = 0;
      if (kKnn && active) src.cut(kr, cd, cj);
      const float2 of = s_posf[active ? kr : 0];
      const F32Test ft = make_f32_test(P, B, of.x, of.y);
      int nshort = -1, vl_cnt = 0;
      unsigned short *vl_out = nullptr;
      if (active && G.vl) nshort = load_candidates(G, a, vl_use, s_nb16, threadIdx.x, vl_out);
      RefAcc A = {};
      double bx = 0.0, by = 0.0;
      int nb = 0;
      ref_particle<kBrute, kKnn, true>(P, src, cur, active, kr, o, ft, s_nb16, A, bx, by, my_pairs, nb, cd, cj, nshort,
                                       vl_out, vl_cnt);
      if (vl_out) G.vl_n[a] = vl_cnt <= kVlMax ? (unsigned char)vl_cnt : kVlOverflow;
      my_nb = max(my_nb, nb);
      if (active) {
        if (F.enabled)
          ref_step_epilogue(P, S, F, a, o, A, bx, by);
        else
          ref_epilogue(P, S, a, o, A, bx, by);
      }
    }
    if (G.vl && !vl_use && threadIdx.x == 0) G.tile_gen[tile] = gen;
  } else {
    // a crowded tile: the same walk over the cell list in global memory
    unsigned *s_nb32 = reinterpret_cast<unsigned *>(rec);
    const GlobalSrc src{P, S};
    for (int base = 0; base < ncore; base += kTileThreads) {
      const int k = base + threadIdx.x;
      int kr = 0, pos = 0, a = 0;
      if (k < ncore) {
        tile_core(B, k, kr, pos);
        a = G.list[pos];
      }
      const bool active = k < ncore && a < P.nf;
      const int as = active ? a : 0;
      const RefOwn o = make_own(P, load_ref_rec(P, S, as));
      GlobalCursor cur;
      cur.list = G.list;
      cur.c.init(P, G, G.cell_of[as]);
      double cd = 0.0;
      int cj = 0;
      if (kKnn && active) src.cut(as, cd, cj);
      const F32Test ft = {};
      RefAcc A = {};
      double bx = 0.0, by = 0.0;
      int nb = 0;
      int vl_none = 0;
      ref_particle<kBrute, kKnn, false>(P, src, cur, active, as, o, ft, s_nb32, A, bx, by, my_pairs, nb, cd, cj, -1,
                                        nullptr, vl_none);
      my_nb = max(my_nb, nb);
      if (active) {
        if (F.enabled)
          ref_step_epilogue(P, S, F, a, o, A, bx, by);
        else
          ref_epilogue(P, S, a, o, A, bx, by);
      }
    }
  }
}

// The REF rate pass: one CTA per storage tile (tile_pass.cuh).  kBrute: the
// wall modes that act on every boundary particle within the radius
// (LeonnardJonesBoundaryForces, MonaghanBoundaryForce) rather than on listed
// pairs.  kKnn: the reference's k-nearest cap (DevParams::knn).
// With F.enabled the pass also applies the step (StepOut): the wall motion
// goes first, grid-strided over the wall slots of F.D, which no CTA of this
// pass reads.
template <bool kBrute, bool kKnn>
__global__ void __launch_bounds__(kTileThreads, 2) k_ref_pass(const DevParams P, const SlotArrays S, const CellGrid G,
                                                           PassStats st, const StepOut F)
{
  extern __shared__ __align__(16) unsigned char smem[];
  if (F.enabled && F.walls) {
    const double t = (*F.d_itime + (F.walls == 2 ? 1 : 0)) * P.dt;
    for (int w = P.nf + blockIdx.x * kTileThreads + threadIdx.x; w < P.n; w += gridDim.x * kTileThreads)
      wall_move_one(P, F.D, F.W, w, t, F.err);
  }
  unsigned my_pairs = 0;
  int my_nb = 0;  // largest in-radius count of this thread's particles
  ref_tile<kBrute, kKnn>(P, S, G, F, blockIdx.x, smem, my_pairs, my_nb);
  pass_stats(st, my_pairs, my_nb);
}

template <bool kBrute, bool kKnn>
uph_status launch_ref(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st, const StepOut &F,
                      cudaStream_t s)
{
  static bool attr_set[64] = {};  // once per device
  int dev = 0;
  UPH_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64 || !attr_set[dev]) {
    UPH_CUDA(cudaFuncSetAttribute(k_ref_pass<kBrute, kKnn>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)ref_smem<kKnn>()));
    if (dev >= 0 && dev < 64) attr_set[dev] = true;
  }
  const int ntiles = P.ntx * (P.ncy / P.tile);
  k_ref_pass<kBrute, kKnn><<<ntiles, kTileThreads, ref_smem<kKnn>(), s>>>(P, S, G, st, F);
  return UPH_OK;
}

uph_status launch_ref_pass(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st,
                           const StepOut &F, cudaStream_t s)
{
  if (P.nf <= 0) return UPH_OK;
  const bool brute = P.boundary_force != 3 && P.boundary_force != 4 && P.boundary_force != 5;
  if (P.knn > 0)
    return brute ? launch_ref<true, true>(P, S, G, st, F, s) : launch_ref<false, true>(P, S, G, st, F, s);
  return brute ? launch_ref<true, false>(P, S, G, st, F, s) : launch_ref<false, false>(P, S, G, st, F, s);
}

// The knn cap's cut of every fluid query: walk the stencil (the global cell
// list, in its order), keep the knn smallest keys (r^2, reference index) of
// the in-radius points (DBL_EPSILON < r^2 < (h h) 4, the own point and
// coincident points excluded, as in SearchNeighbors) in a sorted array, and
// record the largest kept key if more than knn points were in radius.
// One in-radius candidate (r2, reference index) of a query: kept among the
// K smallest keys so far (kd, kj sorted ascending, m of them).
__device__ __forceinline__ void knn_offer(double r2cut, int K, double r2, int ob, double *kd, int *kj, int &m,
                                          int &count)
{
  if (!(r2 < r2cut) || r2 <= DBL_EPSILON) return;
  count++;
  if (m == K && knn_key_le(kd[K - 1], kj[K - 1], r2, ob)) return;  // not among the K smallest
  int i = m < K ? m++ : K - 1;  // the slot the new key may take
  while (i > 0 && !knn_key_le(kd[i - 1], kj[i - 1], r2, ob)) {
    kd[i] = kd[i - 1];
    kj[i] = kj[i - 1];
    i--;
  }
  kd[i] = r2;
  kj[i] = ob;
}

__global__ void __launch_bounds__(128) k_knn_cut(const DevParams P, const SlotArrays S, const CellGrid G,
                                                 const VirtualPoints V)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const int K = P.knn;
  double kd[kKnnMax];
  int kj[kKnnMax];
  int m = 0, count = 0;
  const double xa = S.x[a], ya = S.y[a];
  auto offer = [&](double r2, int ob) { knn_offer(P.r2cut, K, r2, ob, kd, kj, m, count); };
  const int cell = G.cell_of[a];
  NeighbourCursor cur;
  int pos;
  // a first walk only counts the in-radius points: where there are at most
  // K, nothing is cut and the sorted walk is not needed
  int inradius = 0;
  cur.init(P, G, cell);
  while (cur.next(pos)) {
    const int b = G.list[pos];
    if (b == a) continue;
    const double r2 = exact_r2(xa - S.x[b], ya - S.y[b]);
    inradius += (r2 < P.r2cut && r2 > DBL_EPSILON) ? 1 : 0;
  }
  if (V.grid.list) {
    cur.init(P, V.grid, cell);
    while (cur.next(pos)) {
      const int v = V.grid.list[pos];
      const double r2 = exact_r2(xa - V.x[v], ya - V.y[v]);
      inradius += (r2 < P.r2cut && r2 > DBL_EPSILON) ? 1 : 0;
    }
  }
  if (inradius > K) {
    cur.init(P, G, cell);
    while (cur.next(pos)) {
      const int b = G.list[pos];
      if (b == a) continue;
      offer(exact_r2(xa - S.x[b], ya - S.y[b]), S.orig[b]);
    }
    // the virtual mirror particles are points of the reference's search too
    // (reference indices from Nf + Ns + Nb on), though never in a pair
    if (V.grid.list) {
      cur.init(P, V.grid, cell);
      while (cur.next(pos)) {
        const int v = V.grid.list[pos];
        offer(exact_r2(xa - V.x[v], ya - V.y[v]), P.n + v);
      }
    }
  }
  if (count > K) {
    P.kcut_d2[a] = kd[K - 1];
    P.kcut_j[a] = kj[K - 1];
  } else {
    P.kcut_d2[a] = __longlong_as_double(0x7ff0000000000000ll);  // +inf
    P.kcut_j[a] = INT_MAX;
  }
}

void launch_knn_cut(const DevParams &P, const SlotArrays &S, const CellGrid &G, const VirtualPoints &V,
                    cudaStream_t s)
{
  if (P.nf <= 0 || P.knn <= 0) return;
  k_knn_cut<<<(P.nf + 127) / 128, 128, 0, s>>>(P, S, G, V);
}

// ---- stressType 2 (ClassicShearStress, derivatives.c:1686-1721, and
// ViscousForcesTwoStep, :1724-1768) -----------------------------------------------
// Both walk the reference's pair list: every pair sums into both of its
// particles.  Seen from particle a with partner b, d = x_a - x_b and the
// pair's dwcdx = F d (sign included), both roles of a pair give the same
// terms:
//   sigma_a    = -mu sum_b (m_b / rho_b)(rhot_b / rho_a) (dv (x) dw + dw (x) dv)
//                with dv = v_a - vt_b, so sigma_xy = sigma_yx;
//   dv_a/dt   += sum_b m_b (sigma_a / rho_a^2 * rhot_b / rho_b
//                           + sigma_b / rho_b^2 * rhot_a / rho_a) . dw
// (fluid a only; b runs over fluid and wall partners, walls carrying the
// stress of their own fluid pairs).

// the listing rule of the pass (tile_pass.cuh): in the radius, not
// coincident, both below ParticleBoundary, the smaller index a fluid query,
// and with the knn cap the larger index among that query's kept points
template <bool kKnn>
__device__ __forceinline__ bool ref_listed(const DevParams &P, int a, int oa, int b, int ob, double r2)
{
  if (!(r2 < P.r2cut) || r2 <= DBL_EPSILON) return false;
  if (max(oa, ob) >= P.pb || min(oa, ob) >= P.nf) return false;
  if constexpr (kKnn) {
    const int q = ob > oa ? a : b;  // the query's slot: a fluid slot
    return knn_key_le(r2, max(oa, ob), P.kcut_d2[q], P.kcut_j[q]);
  }
  return true;
}

// the poly-7 deconvolution gradient factor F of ref_pair: dwcdx = F d
__device__ __forceinline__ double ref_grad_factor(const DevParams &P, double r2)
{
  const double q2 = r2 * P.inv_h2;
  const double t = fma(-0.25, q2, 1.0);
  const double t2 = t * t, t4 = t2 * t2;
  const double pp7 = fma(fma(fma(fma(fma(fma(305.0, q2, -1106.0), q2, 1912.0), q2, -2912.0), q2, 3712.0), q2, -3584.0), q2, 2048.0);
  return P.dw_alpha_h2 * (t4 * t2 * t) * pp7;
}

template <bool kKnn>
__global__ void __launch_bounds__(128) k_shear_stress(const DevParams P, const SlotArrays S, const CellGrid G)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.n) return;
  const int oa = S.orig[a];
  double sxx = 0.0, sxy = 0.0, syy = 0.0;
  const double ira = S.inv_rho[a];
  if (oa < P.pb) {
    const double xa = S.x[a], ya = S.y[a], ua = S.u[a], va = S.v[a];
    NeighbourCursor cur;
    cur.init(P, G, G.cell_of[a]);
    int k;
    while (cur.next(k)) {
      const int b = G.list[k];
      if (b == a) continue;
      const double dx = xa - S.x[b], dy = ya - S.y[b];
      const double r2 = exact_r2(dx, dy);
      if (!ref_listed<kKnn>(P, a, oa, b, S.orig[b], r2)) continue;
      const double F = ref_grad_factor(P, r2);
      const double dwx = F * dx, dwy = F * dy;
      const double dvx = ua - S.ut[b], dvy = va - S.vt[b];
      // viscosity * reduced volume (m_b / rho_b) rhot_b / rho_a
      const double c = P.mu0 * (S.m[b] * S.inv_rho[b]) * S.rhot[b] * ira;
      sxx -= c * (dvx * dwx + dvx * dwx);
      sxy -= c * (dvx * dwy + dvy * dwx);
      syy -= c * (dvy * dwy + dvy * dwy);
    }
  }
  const double ir2 = ira * ira;
  P.str_xx[a] = sxx * ir2;
  P.str_xy[a] = sxy * ir2;
  P.str_yy[a] = syy * ir2;
}

template <bool kKnn>
__global__ void __launch_bounds__(128) k_viscous_two_step(const DevParams P, const SlotArrays S, const CellGrid G)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.nf) return;
  const int oa = S.orig[a];
  const double xa = S.x[a], ya = S.y[a];
  const double Ca = S.rhot[a] * S.inv_rho[a];
  const double axx = P.str_xx[a], axy = P.str_xy[a], ayy = P.str_yy[a];
  double fx = 0.0, fy = 0.0;
  NeighbourCursor cur;
  cur.init(P, G, G.cell_of[a]);
  int k;
  while (cur.next(k)) {
    const int b = G.list[k];
    if (b == a) continue;
    const double dx = xa - S.x[b], dy = ya - S.y[b];
    const double r2 = exact_r2(dx, dy);
    if (!ref_listed<kKnn>(P, a, oa, b, S.orig[b], r2)) continue;
    const double F = ref_grad_factor(P, r2);
    const double dwx = F * dx, dwy = F * dy;
    const double Cb = S.rhot[b] * S.inv_rho[b];
    const double txx = fma(axx, Cb, P.str_xx[b] * Ca);
    const double txy = fma(axy, Cb, P.str_xy[b] * Ca);
    const double tyy = fma(ayy, Cb, P.str_yy[b] * Ca);
    const double mb = S.m[b];
    fx = fma(mb, fma(txx, dwx, txy * dwy), fx);
    fy = fma(mb, fma(txy, dwx, tyy * dwy), fy);
  }
  S.ax[a] += fx;
  S.ay[a] += fy;
}

void launch_viscous_two_step(const DevParams &P, const SlotArrays &S, const CellGrid &G, cudaStream_t s)
{
  if (P.nf <= 0 || P.stress_type != 2) return;
  if (P.knn > 0) {
    k_shear_stress<true><<<(P.n + 127) / 128, 128, 0, s>>>(P, S, G);
    k_viscous_two_step<true><<<(P.nf + 127) / 128, 128, 0, s>>>(P, S, G);
  } else {
    k_shear_stress<false><<<(P.n + 127) / 128, 128, 0, s>>>(P, S, G);
    k_viscous_two_step<false><<<(P.nf + 127) / 128, 128, 0, s>>>(P, S, G);
  }
}

// ---- particle-packing initialisation (flagInitSimul == 0) ------------------------
// derivatives.c:4279-4288 in place of the physics: the kernel-sum gradient
// of each fluid particle, g_i = V0 sum_pairs dwcdx (both sides, j's with the
// sign flipped: CalculateGradientOfNormalizationFactor, :2977-3012); a
// momentum term that every pair of the particle adds once more,
// -(beta g_i + damp v_i) with beta = 2 g LocalDepth, damp = 0.02
// sqrt(beta / V0), V0 = mass[0] / rho0 (InitializationMomentumEquation,
// :3014-3054); then the hydrostatic reset rho = rho0, p = rho0 g (D - y)
// (InitialDensityAndPressure, :3056-3066) and the selected wall forces as in
// the physics pass.  The other rates stay zero (:3147-3157), and so do the
// fluctuations, which the physics would have set.  CalculateNormalizationFactor
// (:2948-2975) only accumulates into normalizationFactor, which no rate, state
// field or printed column reads; it is not kept.
template <bool kBrute, bool kKnn>
__global__ void __launch_bounds__(128) k_packing_pass(const DevParams P, const SlotArrays S, const CellGrid G,
                                                    PassStats st)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned my_pairs = 0;
  int my_nb = 0;
  if (a < P.nf) {
    const int oa = S.orig[a];
    const double xa = S.x[a], ya = S.y[a], ua = S.u[a], va = S.v[a], ma = S.m[a];
    const int ita = S.itype[a];
    const double cd = kKnn ? P.kcut_d2[a] : 0.0;
    const int cj = kKnn ? P.kcut_j[a] : 0;
    RefAcc A = {};
    double gx = 0.0, gy = 0.0, bx = 0.0, by = 0.0;
    int np = 0;
    NeighbourCursor cur;
    cur.init(P, G, G.cell_of[a]);
    int k;
    while (cur.next(k)) {
      const int b = G.list[k];
      if (b == a) continue;
      const double dx = xa - S.x[b], dy = ya - S.y[b];
      const double r2 = exact_r2(dx, dy);
      if (!(r2 < P.r2cut)) continue;
      const int ob = S.orig[b];
      if (kBrute && ob >= P.b0 && ob < P.b1) brute_wall_force(P, r2, dx, dy, S.m[b], bx, by);
      if (r2 <= DBL_EPSILON) continue;
      my_nb++;
      if (max(oa, ob) >= P.pb) continue;
      const bool isI = ob > oa;
      if constexpr (kKnn) {
        if (!(isI ? knn_key_le(r2, ob, cd, cj) : knn_key_le(r2, oa, P.kcut_d2[b], P.kcut_j[b]))) continue;
      }
      my_pairs += isI;
      const double F = ref_grad_factor(P, r2);
      gx = fma(F, dx, gx);
      gy = fma(F, dy, gy);
      np++;
      if (isI && ita == 1 && S.itype[b] >= 2) wall_pair_force(P, S.itype[b], r2, dx, dy, ua - S.u[b], va - S.v[b], ma, A);
    }
    const double V0 = *P.pack_mass0 / P.rho0;
    const double beta = 2.0 * P.g * P.local_depth;
    const double damp = 0.02 * sqrt(beta / V0);
    const double npd = (double)np;
    A.ax += bx - npd * (beta * (V0 * gx)) - npd * (damp * ua);
    A.ay += by - npd * (beta * (V0 * gy)) - npd * (damp * va);
    S.drho[a] = 0.0;
    S.dp[a] = 0.0;
    S.drho_a[a] = 0.0;
    S.dp_a[a] = 0.0;
    S.ax[a] = A.ax;
    S.ay[a] = A.ay;
    S.ax_a[a] = A.ax_a;
    S.ay_a[a] = A.ay_a;
    S.frho[a] = 0.0;
    S.fp[a] = 0.0;
    S.fu[a] = 0.0;
    S.fv[a] = 0.0;
    S.rho[a] = P.rho0;
    S.p[a] = P.rho0 * P.g * (P.local_depth - ya);
  }
  pass_stats(st, my_pairs, my_nb);
}

uph_status launch_packing_pass(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st,
                               cudaStream_t s)
{
  if (P.nf <= 0) return UPH_OK;
  const bool brute = P.boundary_force != 3 && P.boundary_force != 4 && P.boundary_force != 5;
  const int blocks = (P.nf + 127) / 128;
  if (P.knn > 0) {
    if (brute) k_packing_pass<true, true><<<blocks, 128, 0, s>>>(P, S, G, st);
    else k_packing_pass<false, true><<<blocks, 128, 0, s>>>(P, S, G, st);
  } else {
    if (brute) k_packing_pass<true, false><<<blocks, 128, 0, s>>>(P, S, G, st);
    else k_packing_pass<false, false><<<blocks, 128, 0, s>>>(P, S, G, st);
  }
  return UPH_OK;
}

__global__ void k_rcp_selftest(const double *__restrict__ x, double *__restrict__ y, int64_t n)
{
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    y[k] = rcp_nr(x[k]);
}

}  // namespace uph

extern "C" uph_status uph_rcp_selftest(const double *x, double *y, int64_t n, void *stream)
{
  if (n < 0 || (n > 0 && (!x || !y))) return uph::fail(UPH_BAD_ARG, "uph_rcp_selftest: bad arguments");
  if (n == 0) return UPH_OK;
  const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  uph::k_rcp_selftest<<<blocks, 256, 0, (cudaStream_t)stream>>>(x, y, n);
  UPH_CUDA(cudaGetLastError());
  return UPH_OK;
}
