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
// Execution: one thread per fluid slot.  Each thread first walks its 5 x 5
// block of half-radius cells with only the exact distance test and lists the
// in-radius partners in shared memory (kNbChunk at a time); then the warp runs the heavy FP64 pair
// arithmetic over those lists.  The lists have nearly equal lengths, so the
// lanes of a warp stay converged in the expensive loop instead of idling while
// their neighbours reject out-of-radius candidates.
#include "pass_common.cuh"

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

// LeonnardJonesBoundaryForces (mode 1, derivatives.c:1184-1211) and
// MonaghanBoundaryForce (default mode, :1919-1953): every fluid particle
// against every boundary particle, no pair-list filter.
__device__ __forceinline__ void brute_wall_force(const DevParams &P, double r2, double dxa, double dya, double mb,
                                                 double &fx, double &fy)
{
  if (P.boundary_force == 1) {
    const double r0 = P.dx;
    if (r2 < r0 * r0) {
      double rr = r0 / sqrt(r2);
      rr *= rr;
      rr *= rr;
      const double pb = P.lj_coeff * rr * (rr * rr - 1.) / r2;
      fx += pb * dxa;
      fy += pb * dya;
    }
  } else {
    const double r = sqrt(r2);
    const double q = r / P.h;
    double phi = 0.0;
    if (q >= 0.0 && q < 2.0) {
      const double t = 2.0 - q;
      phi = 0.125 * (1.0 + 1.5 * q) * t * t * t;
    }
    const double gama = P.mach_c * P.mach_c / (P.rho0 * P.dx * P.dy);
    const double c = gama * phi * mb / r2;
    fx += c * dxa;
    fy += c * dya;
  }
}

__global__ void __launch_bounds__(kPassThreads, 4) k_ref_pass(const DevParams P, const SlotArrays S, const CellGrid G,
                                                           PassStats st)
{
  __shared__ unsigned s_nb[kNbChunk][kPassThreads];
  const int tid = threadIdx.x;
  const int a = blockIdx.x * blockDim.x + tid;
  const bool active = a < P.nf;
  unsigned my_pairs = 0;
  int my_nb = 0;
  const int as = active ? a : 0;
  const double xa = S.x[as], ya = S.y[as];
  const double ua = S.u[as], va = S.v[as], uta = S.ut[as], vta = S.vt[as];
  const double rhoa = S.rho[as], rhota = S.rhot[as], pa = S.p[as], ma = S.m[as];
  const double ira = S.inv_rho[as], irta = S.inv_rhot[as];
  const int oa = S.orig[as], ita = S.itype[as];
  const double Pa = P.rho0c2 + P.gamma * pa;
  const double ira2 = ira * ira;
  const double gk = P.gamma * P.kappa;
  const bool brute_walls = P.boundary_force != 3 && P.boundary_force != 4 && P.boundary_force != 5;
  RefAcc A = {};
  double bx = 0.0, by = 0.0;  // mode-1 / default wall force (dvdt only)

  NeighbourCursor cur;
  cur.init(P, G, G.cell_of[as]);
  bool more = active;
  while (__any_sync(0xffffffffu, more)) {
    // phase 1: list up to kNbChunk partners (distance test and pair filter only)
    const int cnt = list_partners(P, S, G, cur, more, a, oa, xa, ya, s_nb, tid, my_pairs, my_nb,
                                  [&](int b, int ob, double r2, double dxa, double dya) {
                                    if (brute_walls && ob >= P.b0 && ob < P.b1)
                                      brute_wall_force(P, r2, dxa, dya, S.m[b], bx, by);
                                  });
    __syncwarp();
    // phase 2: the pair terms
    for (int e = 0; e < cnt; e++) {
      const unsigned ent = s_nb[e][tid];
      const int b = (int)(ent & ~kRoleI);
      const bool isI = (ent & kRoleI) != 0;
      const double dxa = xa - S.x[b], dya = ya - S.y[b];
      const double r2 = exact_r2(dxa, dya);
      const double ub = S.u[b], vb = S.v[b], utb = S.ut[b], vtb = S.vt[b];
      const double rhob = S.rho[b], rhotb = S.rhot[b], pb = S.p[b], ptb = S.pt[b], mb = S.m[b];
      const double irb = S.inv_rho[b], irtb = S.inv_rhot[b];

      // poly-7 convolution W and deconvolution gradient factor: functions of q^2 only
      const double q2 = r2 * P.inv_h2;
      const double t = fma(-0.25, q2, 1.0);
      const double t2 = t * t, t4 = t2 * t2;
      const double t7 = t4 * t2 * t, t8 = t4 * t4;
      const double pp = fma(fma(fma(fma(fma(fma(305.0, q2, -628.0), q2, 1184.0), q2, -1984.0), q2, 2816.0), q2, -3072.0), q2, 2048.0);
      const double pp7 = fma(fma(fma(fma(fma(fma(305.0, q2, -1106.0), q2, 1912.0), q2, -2912.0), q2, 3712.0), q2, -3584.0), q2, 2048.0);
      const double W = P.w_alpha * t8 * pp;
      const double F = P.dw_alpha * P.inv_h2 * t7 * pp7;
      const double gx = F * dxa, gy = F * dya;

      const double Pb = fma(P.gamma, pb, P.rho0c2);
      const double Vb = mb * irb;
      const double ms = isI ? mb : ma;
      const double rhosum = ira + irb;
      const double inv_r2e = rcp_nr(r2 + P.eta2);
      const double nu = (dxa * gx + dya * gy) * inv_r2e;
      const double ep = 4.0 * Pa * rcp_nr(Pa + Pb);

      // predictor density
      const double pdx = isI ? (ua - utb) : (uta - ub);
      const double pdy = isI ? (va - vtb) : (vta - vb);
      A.drho_a += ms * (pdx * gx + pdy * gy);
      // predictor pressure
      const double dux = ua - ub, duy = va - vb;
      const double vdw = dux * gx + duy * gy;
      const double msb = ms * irb;
      A.dp_a += (mb * ira) * Pa * vdw + gk * msb * (pa - pb) * nu * ep - P.kappa * Pa * msb * (rhoa - rhob) * rhosum * nu;
      // predictor pressure gradient
      const double pij_p = pa * ira2 + pb * irb * irb;
      A.ax_a -= mb * pij_p * gx;
      A.ay_a -= mb * pij_p * gy;
      // fluctuations
      A.frho -= Vb * (rhoa - rhob) * W;
      A.fp -= Vb * (pa - pb) * W;
      const double cfv = isI ? (ma * irtb - mb * irta) * W : 0.0;
      A.fu += dux * cfv;
      A.fv += duy * cfv;
      // continuity
      const double vdwt = (ua - utb) * gx + (va - vtb) * gy;
      const double Vr = Vb * rhotb;
      A.drho += Vr * vdwt;
      // rate-form Tait with diffusion
      A.dp += Vr * ira * Pa * vdwt + gk * Vb * (pa - ptb) * nu * ep - P.kappa * Pa * Vb * (rhoa - rhotb) * rhosum * nu;
      // pressure gradient
      const double pij = pa * rhotb * ira2 * irb + pb * rhota * irb * irb * ira;
      A.ax -= mb * pij * gx;
      A.ay -= mb * pij * gy;
      // deviatoric viscous stress
      if (P.stress_type == 1) {
        const double meff = 2.0 * P.mu0 * rcp_nr(rhosum);
        const double s00 = (-dxa) * dux - (-dya) * duy;
        const double s01 = (-dxa) * duy + (-dya) * dux;
        const double sgx = s00 * gx + s01 * gy;
        const double sgy = s01 * gx - s00 * gy;
        const double base = mb * meff * inv_r2e;
        const double D = rhotb * ira2 * irb - rhota * irb * irb * ira;
        const double sD = (isI ? base : -base) * D;
        A.ax += sD * sgx;
        A.ay += sD * sgy;
        const double Dp = base * (ira2 + irb * irb);
        A.ax_a += Dp * sgx;
        A.ay_a += Dp * sgy;
      }
      // wall forces: only pairs whose i is this fluid particle
      if (isI && ita == 1) {
        const int itb = S.itype[b];
        if (itb >= 2) wall_pair_force(P, itb, r2, dxa, dya, dux, duy, ma, A);
      }
    }
    __syncwarp();
  }
  if (active) {
    A.ax += bx;
    A.ay += by;
    if (P.gravity_flag == 1) {
      A.ay -= P.g;
      A.ay_a -= P.g;
    }
    if (P.moving_boundary == 1 && P.wave_absorption == 1) A.ax -= S.sponge[a] * ua;
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
    S.pressure[a] = P.B * (pow(rhoa / P.rho0, P.gamma) - 1.0);
  }
  // pass statistics: one atomic per warp
  const unsigned wp = __reduce_add_sync(0xffffffffu, my_pairs);
  const int wn = (int)__reduce_max_sync(0xffffffffu, (unsigned)my_nb);
  if ((threadIdx.x & 31) == 0) {
    if (wp) atomicAdd(st.niac, (unsigned long long)wp);
    if (wn) atomicMax(st.max_nb, wn);
  }
}

void launch_ref_pass(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st, cudaStream_t s)
{
  if (P.nf <= 0) return;
  k_ref_pass<<<(P.nf + kPassThreads - 1) / kPassThreads, kPassThreads, 0, s>>>(P, S, G, st);
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
