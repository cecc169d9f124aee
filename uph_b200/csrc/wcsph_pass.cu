// The fused rate pass of the WCSPH profile on the same cell list and pair
// set as the REF pass:
//   drho_a = sum_b m_b (v_a - v_b) . grad_a W_ab
//   dv_a   = -sum_b m_b (p_a/rho_a^2 + p_b/rho_b^2 + Pi_ab) grad_a W_ab + g + walls
//   Pi_ab  = -alpha c0 h (v_ab . x_ab) / (r^2 + 0.01 h^2) / rhobar_ab   if v_ab . x_ab < 0
// with the reference's cubic spline Kernel() (derivatives.c:44-66) and the
// algebraic Tait pressure (derivatives.c:1674-1682) evaluated before the pass.
// Monaghan's viscosity (Monaghan 1992, Annu. Rev. Astron. Astrophys. 30:543,
// beta = 0) has no counterpart in the reference.  Wall forces are the
// reference's (derivatives.c:2396-2449 and the other selectBoundaryForce
// modes), in FP64.
//
// Real = double: everything in FP64.  Real = float: the pair arithmetic and
// the per-particle sums run in FP32 from FP64 differences of positions and
// velocities (taken before rounding, so small separations keep their
// precision); the pair test itself stays the exact FP64 predicate so both
// precisions see the same pairs.  The partner's m, p / rho^2 and rho come
// from one packed FP32 load (SlotArrays::pk, rounded once from FP64 where
// 1/rho is refreshed) instead of four FP64 loads.
//
// Execution as in the REF pass: a cheap listing phase (distance test only)
// per thread into shared memory, then the pair arithmetic over the lists.
#include "pass_common.cuh"

namespace uph {

template <typename Real>
__device__ __forceinline__ Real rcp_real(Real x);
template <>
__device__ __forceinline__ double rcp_real<double>(double x) { return rcp_nr(x); }
template <>
__device__ __forceinline__ float rcp_real<float>(float x) { return __frcp_rn(x); }

template <typename Real>
__device__ __forceinline__ Real sqrt_real(Real x);
template <>
__device__ __forceinline__ double sqrt_real<double>(double x) { return sqrt(x); }
template <>
__device__ __forceinline__ float sqrt_real<float>(float x) { return __fsqrt_rn(x); }

// selectBoundaryForce modes that act on listed pairs (i side = this fluid particle)
__device__ __forceinline__ void wcsph_wall_pair(const DevParams &P, int itb, double r2d, double dxd, double dyd,
                                                double dud, double dvd, double ma, double &wx, double &wy)
{
  const double rr = sqrt(r2d);
  if (P.boundary_force == 3 && (itb == 2 || itb == 3 || itb == 5)) {
    const double r0 = 3.0 * P.dx;
    if (rr < r0) {
      const double rv = dxd * dud + dyd * dvd;
      const double c1 = P.k_spring * (r0 - rr) / (rr * ma);
      const double c2 = P.c_damp * rv / (rr * rr * ma);
      wx -= c1 * dxd + c2 * dxd;
      wy -= c1 * dyd + c2 * dyd;
    }
  } else if (P.boundary_force == 4 && (itb == 2 || itb == 3) && rr < P.dx) {
    const double norm = 7.0 / (64.0 * 3.142 * P.h * P.h);
    const double qq = rr / P.h;
    double phi = 0.0;
    if (qq < 2.0) {
      const double t = 2.0 - qq;
      phi = norm * (1.0 + 2.0 * qq) * (t * t) * (t * t);
    }
    const double c = P.mach_c * P.mach_c / 5.0 * phi / ((rr - P.dx / 5.0) * rr);
    wx += c * dxd;
    wy += c * dyd;
  } else if (P.boundary_force == 5 && itb == 2 && rr < P.dx) {
    wx -= (P.k_spring * dxd + P.c_damp * dud) / ma;
    wy -= (P.k_spring * dyd + P.c_damp * dvd) / ma;
  }
}

// modes 1 / default: every boundary particle, no pair filter (FP64, as the REF pass)
__device__ __forceinline__ void wcsph_wall_brute(const DevParams &P, double r2d, double dxd, double dyd, double mb,
                                                 double &wx, double &wy)
{
  if (P.boundary_force == 1) {
    const double r0 = P.dx;
    if (r2d < r0 * r0) {
      double rr = r0 / sqrt(r2d);
      rr *= rr;
      rr *= rr;
      const double pb = P.lj_coeff * rr * (rr * rr - 1.) / r2d;
      wx += pb * dxd;
      wy += pb * dyd;
    }
  } else {
    const double rr = sqrt(r2d), q = rr / P.h;
    double phi = 0.0;
    if (q < 2.0) {
      const double t = 2.0 - q;
      phi = 0.125 * (1.0 + 1.5 * q) * t * t * t;
    }
    const double c = P.mach_c * P.mach_c / (P.rho0 * P.dx * P.dy) * phi * mb / r2d;
    wx += c * dxd;
    wy += c * dyd;
  }
}

template <typename Real>
__global__ void __launch_bounds__(kPassThreads, 5) k_wcsph_pass(const DevParams P, const SlotArrays S, const CellGrid G,
                                                             PassStats st)
{
  __shared__ unsigned s_nb[kNbChunk][kPassThreads];
  const int tid = threadIdx.x;
  const int a = blockIdx.x * blockDim.x + tid;
  const bool active = a < P.nf;
  unsigned my_pairs = 0;
  int my_nb = 0;
  const int as = active ? a : 0;
  const double xa = S.x[as], ya = S.y[as], ua = S.u[as], va = S.v[as];
  const double ma_d = S.m[as];
  // FP32 pair arithmetic reads the packed operands written with 1/rho
  constexpr bool kPacked = sizeof(Real) == sizeof(float);
  Real pa_over, rhoa;
  if constexpr (kPacked) {
    const float4 k = S.pk[as];
    pa_over = k.y;
    rhoa = k.z;
  } else {
    const Real ira = (Real)S.inv_rho[as];
    pa_over = (Real)S.p[as] * ira * ira;
    rhoa = (Real)S.rho[as];
  }
  const int oa = S.orig[as], ita = S.itype[as];
  const Real h = (Real)P.h, inv_h = (Real)P.inv_h, inv_h2 = (Real)P.inv_h2;
  const Real sigma = (Real)P.cs_alpha;
  const Real eta2 = (Real)P.eta2, ac = (Real)P.av_alpha_c0;
  const bool brute_walls = P.boundary_force != 3 && P.boundary_force != 4 && P.boundary_force != 5;
  Real drho = 0, ax = 0, ay = 0;
  double wx = 0.0, wy = 0.0;  // wall forces, FP64 like the reference

  NeighbourCursor cur;
  cur.init(P, G, G.cell_of[as]);
  bool more = active;
  while (__any_sync(0xffffffffu, more)) {
    const int cnt = list_partners(P, S, G, cur, more, a, oa, xa, ya, s_nb, tid, my_pairs, my_nb,
                                  [&](int b, int ob, double r2d, double dxd, double dyd) {
                                    if (brute_walls && ob >= P.b0 && ob < P.b1)
                                      wcsph_wall_brute(P, r2d, dxd, dyd, S.m[b], wx, wy);
                                  });
    __syncwarp();
    for (int e = 0; e < cnt; e++) {
      const unsigned ent = s_nb[e][tid];
      const int b = (int)(ent & ~kRoleI);
      const bool isI = (ent & kRoleI) != 0;
      const double dxd = xa - S.x[b], dyd = ya - S.y[b];
      const double dud = ua - S.u[b], dvd = va - S.v[b];
      const Real dx = (Real)dxd, dy = (Real)dyd, du = (Real)dud, dv = (Real)dvd;
      // partner operands: FP64 fields, or the packed FP32 copy (one 16-byte load)
      Real mb, pb_over, rhob;
      if constexpr (kPacked) {
        const float4 k = S.pk[b];
        mb = k.x;
        pb_over = k.y;
        rhob = k.z;
      } else {
        const Real irb = (Real)S.inv_rho[b];
        mb = (Real)S.m[b];
        pb_over = (Real)S.p[b] * irb * irb;
        rhob = (Real)S.rho[b];
      }
      const Real r2 = dx * dx + dy * dy;
      const Real r = sqrt_real<Real>(r2);
      const Real q = r * inv_h;
      Real F;
      if (q < (Real)1) {
        F = sigma * ((Real)-3 + (Real)2.25 * q) * inv_h2;
      } else {
        const Real t = (Real)2 - q;
        F = -sigma * (Real)0.75 * t * t * inv_h * rcp_real<Real>(r);
      }
      const Real gx = F * dx, gy = F * dy;
      drho += mb * (du * gx + dv * gy);
      const Real vr = du * dx + dv * dy;
      Real pi_ab = 0;
      if (vr < (Real)0) {
        const Real mu = h * vr * rcp_real<Real>(r2 + eta2);
        pi_ab = -ac * mu * rcp_real<Real>((Real)0.5 * (rhoa + rhob));
      }
      const Real pij = pa_over + pb_over + pi_ab;
      ax -= mb * pij * gx;
      ay -= mb * pij * gy;
      if (isI && ita == 1) {
        const int itb = S.itype[b];
        if (itb >= 2) wcsph_wall_pair(P, itb, exact_r2(dxd, dyd), dxd, dyd, dud, dvd, ma_d, wx, wy);
      }
    }
    __syncwarp();
  }
  if (active) {
    double axd = (double)ax + wx, ayd = (double)ay + wy;
    if (P.gravity_flag == 1) ayd -= P.g;
    if (P.moving_boundary == 1 && P.wave_absorption == 1) axd -= S.sponge[a] * ua;
    S.drho[a] = (double)drho;
    S.dp[a] = 0.0;
    S.ax[a] = axd;
    S.ay[a] = ayd;
    S.drho_a[a] = (double)drho;
    S.dp_a[a] = 0.0;
    S.ax_a[a] = axd;
    S.ay_a[a] = ayd;
    S.frho[a] = 0.0;
    S.fp[a] = 0.0;
    S.fu[a] = 0.0;
    S.fv[a] = 0.0;
  }
  const unsigned wp = __reduce_add_sync(0xffffffffu, my_pairs);
  const int wn = (int)__reduce_max_sync(0xffffffffu, (unsigned)my_nb);
  if ((threadIdx.x & 31) == 0) {
    if (wp) atomicAdd(st.niac, (unsigned long long)wp);
    if (wn) atomicMax(st.max_nb, wn);
  }
}

void launch_wcsph_pass(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st, cudaStream_t s)
{
  if (P.nf <= 0) return;
  const int blocks = (P.nf + kPassThreads - 1) / kPassThreads;
  if (P.precision == UPH_PREC_FP32_PAIR)
    k_wcsph_pass<float><<<blocks, kPassThreads, 0, s>>>(P, S, G, st);
  else
    k_wcsph_pass<double><<<blocks, kPassThreads, 0, s>>>(P, S, G, st);
}

}  // namespace uph
