// The fused rate pass of the WCSPH profile on the same cell list and pair
// set as the REF pass:
//   drho_a = sum_b m_b (v_a - v_b) . grad_a W_ab
//   dv_a   = -sum_b m_b (p_a/rho_a^2 + p_b/rho_b^2 + Pi_ab) grad_a W_ab + g + walls
//   Pi_ab  = -alpha c0 h (v_ab . x_ab) / (r^2 + 0.01 h^2) / rhobar_ab   if v_ab . x_ab < 0
// with the reference's cubic spline Kernel() (derivatives.c:44-66) and the
// algebraic Tait pressure (derivatives.c:1674-1682) evaluated before the pass.
// Monaghan's viscosity (Monaghan 1992, Annu. Rev. Astron. Astrophys. 30:543,
// beta = 0) has no counterpart in the reference.
//
// Real = double: everything in FP64.  Real = float: the pair arithmetic and
// the per-particle sums run in FP32 from FP64 differences of positions and
// velocities (computed before rounding, so the small separations keep their
// precision); the pair test itself stays the exact FP64 predicate so both
// precisions see the same pairs.
#include <float.h>

#include "uph_internal.cuh"

namespace uph {

__device__ __forceinline__ double exact_r2w(double dx, double dy)
{
  return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

template <typename Real>
__global__ void __launch_bounds__(128) k_wcsph_pass(const DevParams P, const SlotArrays S, const CellGrid G,
                                                    PassStats st)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = a < P.nf;
  unsigned long long my_pairs = 0;
  int my_nb = 0;
  if (active) {
    const double xa = S.x[a], ya = S.y[a], ua = S.u[a], va = S.v[a];
    const double ma_d = S.m[a];
    const Real ira = (Real)S.inv_rho[a];
    const Real pa_over = (Real)S.p[a] * ira * ira;
    const Real rhoa = (Real)S.rho[a];
    const int oa = S.orig[a], ita = S.itype[a];
    const Real h = (Real)P.h, inv_h = (Real)P.inv_h, inv_h2 = (Real)P.inv_h2;
    const Real sigma = (Real)P.cs_alpha;
    const Real eta2 = (Real)P.eta2, ac = (Real)P.av_alpha_c0;
    const bool brute_walls = (P.boundary_force == 1) || (P.boundary_force != 3 && P.boundary_force != 4 &&
                                                         P.boundary_force != 5);
    Real drho = 0, ax = 0, ay = 0;
    double wx = 0.0, wy = 0.0;  // wall forces, FP64 like the reference
    const int c = G.cell_of[a];
    const int cx = c % P.ncx, cy = c / P.ncx;
    for (int yy = max(cy - 1, 0); yy <= min(cy + 1, P.ncy - 1); yy++) {
      for (int xx = max(cx - 1, 0); xx <= min(cx + 1, P.ncx - 1); xx++) {
        const int cc = yy * P.ncx + xx;
        const int k1 = G.start[cc + 1];
        for (int k = G.start[cc]; k < k1; k++) {
          const int b = G.list[k];
          if (b == a) continue;
          const double dxd = xa - S.x[b], dyd = ya - S.y[b];
          const double r2d = exact_r2w(dxd, dyd);
          if (!(r2d < P.r2cut)) continue;
          const int ob = S.orig[b];
          if (brute_walls && ob >= P.b0 && ob < P.b1) {
            // modes 1 / default, same arithmetic as the REF pass
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
              const double c2 = P.mach_c * P.mach_c / (P.rho0 * P.dx * P.dy) * phi * S.m[b] / r2d;
              wx += c2 * dxd;
              wy += c2 * dyd;
            }
          }
          if (r2d <= DBL_EPSILON) continue;
          my_nb++;
          const bool isI = ob > oa;
          if (max(oa, ob) >= P.pb) continue;
          if (isI) my_pairs++;

          const double dud = ua - S.u[b], dvd = va - S.v[b];
          const Real dx = (Real)dxd, dy = (Real)dyd, du = (Real)dud, dv = (Real)dvd;
          const Real r2 = (Real)r2d;
          const Real r = sqrt(r2);
          const Real q = r * inv_h;
          Real F;
          if (q < (Real)1) {
            F = sigma * ((Real)-3 + (Real)2.25 * q) * inv_h2;
          } else {
            const Real t = (Real)2 - q;
            F = -sigma * (Real)0.75 * t * t * inv_h / r;
          }
          const Real gx = F * dx, gy = F * dy;
          const Real mb = (Real)S.m[b];
          const Real irb = (Real)S.inv_rho[b];
          drho += mb * (du * gx + dv * gy);
          const Real vr = du * dx + dv * dy;
          Real pi_ab = 0;
          if (vr < (Real)0) {
            const Real mu = h * vr / (r2 + eta2);
            pi_ab = -ac * mu / ((Real)0.5 * (rhoa + (Real)S.rho[b]));
          }
          const Real pij = pa_over + (Real)S.p[b] * irb * irb + pi_ab;
          ax -= mb * pij * gx;
          ay -= mb * pij * gy;
          if (isI && ita == 1) {
            const int itb = S.itype[b];
            const double rr = sqrt(r2d);
            if (P.boundary_force == 3 && (itb == 2 || itb == 3 || itb == 5)) {
              const double r0 = 3.0 * P.dx;
              if (rr < r0) {
                const double rv = dxd * dud + dyd * dvd;
                const double c1 = P.k_spring * (r0 - rr) / (rr * ma_d);
                const double c2 = P.c_damp * rv / (rr * rr * ma_d);
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
              const double cc2 = P.mach_c * P.mach_c / 5.0 * phi / ((rr - P.dx / 5.0) * rr);
              wx += cc2 * dxd;
              wy += cc2 * dyd;
            } else if (P.boundary_force == 5 && itb == 2 && rr < P.dx) {
              wx -= (P.k_spring * dxd + P.c_damp * dud) / ma_d;
              wy -= (P.k_spring * dyd + P.c_damp * dvd) / ma_d;
            }
          }
        }
      }
    }
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
  const unsigned long long wp = __reduce_add_sync(0xffffffffu, (unsigned)my_pairs);
  const int wn = (int)__reduce_max_sync(0xffffffffu, (unsigned)my_nb);
  if ((threadIdx.x & 31) == 0) {
    if (wp) atomicAdd(st.niac, wp);
    if (wn) atomicMax(st.max_nb, wn);
  }
}

void launch_wcsph_pass(const DevParams &P, const SlotArrays &S, const CellGrid &G, PassStats st, cudaStream_t s)
{
  if (P.nf <= 0) return;
  if (P.precision == UPH_PREC_FP32_PAIR)
    k_wcsph_pass<float><<<(P.nf + 127) / 128, 128, 0, s>>>(P, S, G, st);
  else
    k_wcsph_pass<double><<<(P.nf + 127) / 128, 128, 0, s>>>(P, S, G, st);
}

}  // namespace uph
